"""Python binding of the engine's C ABI (``include/flowlb.h``).

``Solver`` mirrors FlowLB's solver boundary (``src/cuda/runCuda.cuh:25-38``):
construct from geometry flags and options, ``step(n)``, read back density,
velocity, fill fraction and flags.  It is a thin ctypes layer over
``libflowlb.so``; there is no CPU path: if the library cannot be loaded or no
CUDA device is present, construction raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("FLOWLB_LIB", os.path.join(HERE, "libflowlb.so"))

FIELD_F, FIELD_RHO, FIELD_U, FIELD_FLAGS, FIELD_MASS, FIELD_EXCESS, FIELD_PHI = range(7)
BB_IMPLICIT, BB_HALFWAY = 0, 1
FS_REFERENCE, FS_CONSERVATIVE = 0, 1
ARITH_REFERENCE, ARITH_FUSED = 0, 1

STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported",
          5: "I/O error", 6: "non-finite populations", 7: "no CUDA device"}

# Every symbol the header declares; tests check the library exports them all.
EXPORTS = [
    "flb_case_desc_init", "flb_create", "flb_reset", "flb_destroy", "flb_step", "flb_sync", "flb_get_time",
    "flb_set_step_mode", "flb_get_step_mode", "flb_set_wait_limit",
    "flb_set_stream", "flb_get_stream", "flb_field_info", "flb_read_field", "flb_write_field", "flb_total_mass",
    "flb_total_mass_noalloc", "flb_cell_counts", "flb_check_finite", "flb_run_pass", "flb_profile_steps", "flb_profile_phases", "flb_launch_count", "flb_save_checkpoint",
    "flb_load_checkpoint", "flb_last_error", "flb_status_string", "flb_version",
    "flb_batch_create", "flb_batch_step", "flb_batch_sync", "flb_batch_reset", "flb_batch_read_field",
    "flb_batch_info", "flb_batch_set_launch", "flb_batch_set_wait_limit", "flb_batch_tune", "flb_batch_destroy",
    "flb_batch_last_error",
    "flb_adjoint_desc_init", "flb_adjoint_create", "flb_adjoint_set_porosity", "flb_adjoint_set_force",
    "flb_adjoint_forward", "flb_adjoint_backward", "flb_adjoint_timing", "flb_adjoint_destroy",
    "flb_adjoint_last_error",
    "flb_setup_from_files", "flb_setup_free", "flb_setup_initial_flags", "flb_setup_write_mesh_vti",
    "flb_create_from_files", "flb_write_vti", "flb_write_vti_series", "flb_run_from_files",
    "flb_viz_velocity", "flb_viz_shade", "flb_viz_isoline",
]


class CaseDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("flags", C.c_void_p), ("free_surface", C.c_int32),
        ("precision", C.c_int32), ("mass_precision", C.c_int32), ("collision", C.c_int32),
        ("subgrid", C.c_int32), ("use_volumetric_force", C.c_int32), ("tau", C.c_float), ("fx", C.c_float),
        ("fy", C.c_float), ("bounce_back", C.c_int32), ("fs_mode", C.c_int32), ("f16_scale", C.c_float),
        ("device", C.c_int32), ("stream", C.c_void_p), ("inlet_ux", C.c_double), ("inlet_uy", C.c_double),
        ("kernel_variant", C.c_int32), ("u_max", C.c_float), ("arithmetic", C.c_int32),
    ]


class AdjointDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("flags", C.c_void_p), ("porosity", C.c_void_p),
        ("precision", C.c_int32), ("tau", C.c_double), ("gx", C.c_double), ("gy", C.c_double),
        ("steps", C.c_uint64), ("window", C.c_uint64), ("checkpoint_every", C.c_uint32), ("device", C.c_int32),
        ("stream", C.c_void_p),
    ]


class SetupStruct(C.Structure):
    _fields_ = [
        ("nx", C.c_uint32), ("ny", C.c_uint32), ("x_min", C.c_double), ("y_min", C.c_double),
        ("z_min", C.c_double), ("spacing", C.c_double), ("flags", C.c_void_p), ("desc", CaseDesc),
        ("time_steps", C.c_uint64), ("save_every", C.c_uint64), ("time_simulation", C.c_float),
        ("time_save", C.c_float), ("nu_lattice", C.c_float), ("length_to_si", C.c_double),
        ("time_to_si", C.c_double), ("mass_to_si", C.c_double), ("velocity_to_si", C.c_double),
        ("rho_to_si", C.c_double), ("graphics_api", C.c_int32), ("reference_precision", C.c_int32),
        ("cuda_block", C.c_uint32 * 3), ("error", C.c_char * 256),
    ]


VTI_UINT8, VTI_FLOAT32, VTI_FLOAT64 = 0, 1, 2
VIZ_UX, VIZ_UY, VIZ_MAGNITUDE, VIZ_PRESSURE = 0, 1, 2, 3
BATCH_CLUSTER, BATCH_TEAM, BATCH_VECTOR, BATCH_STREAMS = 0, 1, 4, 8
TUNE_PERSISTENT, TUNE_STREAMS = 1, 2
STEP_AUTO, STEP_KERNELS, STEP_PERSISTENT = 0, 1, 2


class VtiField(C.Structure):
    _fields_ = [("name", C.c_char_p), ("type", C.c_int32), ("components", C.c_int32), ("data", C.c_void_p),
                ("to_si", C.c_double), ("flip_y", C.c_int32)]


class RunInfo(C.Structure):
    _fields_ = [("steps", C.c_uint64), ("files", C.c_uint32), ("directory", C.c_char * 512),
                ("error", C.c_char * 256)]


class FlowLBError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libflowlb.so and declares the C signatures.  Raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; "
                                f"g.build()'` or `make -C flowlb_b200/csrc`")
    L = C.CDLL(path)
    H = C.c_void_p
    sig = {
        "flb_case_desc_init": (None, [C.POINTER(CaseDesc)]),
        "flb_create": (C.c_int, [C.POINTER(CaseDesc), C.POINTER(H)]),
        "flb_reset": (C.c_int, [H, C.c_void_p]),
        "flb_destroy": (C.c_int, [H]),
        "flb_step": (C.c_int, [H, C.c_uint64]),
        "flb_sync": (C.c_int, [H]),
        "flb_get_time": (C.c_int, [H, C.POINTER(C.c_uint64)]),
        "flb_set_stream": (C.c_int, [H, C.c_void_p]),
        "flb_set_step_mode": (C.c_int, [H, C.c_int]),
        "flb_get_step_mode": (C.c_int, [H, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
        "flb_set_wait_limit": (C.c_int, [H, C.c_uint32]),
        "flb_get_stream": (C.c_int, [H, C.POINTER(C.c_void_p)]),
        "flb_field_info": (C.c_int, [H, C.c_int, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
        "flb_read_field": (C.c_int, [H, C.c_int, C.c_void_p, C.c_int]),
        "flb_write_field": (C.c_int, [H, C.c_int, C.c_void_p, C.c_int]),
        "flb_total_mass": (C.c_int, [H, C.POINTER(C.c_double)]),
        "flb_total_mass_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_int,
                                             C.c_void_p, C.c_void_p]),
        "flb_cell_counts": (C.c_int, [H, C.POINTER(C.c_uint64)]),
        "flb_check_finite": (C.c_int, [H]),
        "flb_run_pass": (C.c_int, [H, C.c_int]),
        "flb_profile_steps": (C.c_int, [H, C.c_uint64, C.POINTER(C.c_double)]),
        "flb_profile_phases": (C.c_int, [H, C.c_uint64, C.POINTER(C.c_double)]),
        "flb_launch_count": (C.c_int, [H, C.POINTER(C.c_uint64)]),
        "flb_save_checkpoint": (C.c_int, [H, C.c_char_p]),
        "flb_load_checkpoint": (C.c_int, [H, C.c_char_p]),
        "flb_last_error": (C.c_char_p, [H]),
        "flb_status_string": (C.c_char_p, [C.c_int]),
        "flb_version": (C.c_char_p, []),
        "flb_batch_create": (C.c_int, [C.POINTER(CaseDesc), C.c_uint32, C.c_int, C.POINTER(H)]),
        "flb_batch_step": (C.c_int, [H, C.c_uint64]),
        "flb_batch_sync": (C.c_int, [H]),
        "flb_batch_reset": (C.c_int, [H]),
        "flb_batch_read_field": (C.c_int, [H, C.c_uint32, C.c_int, C.c_void_p, C.c_int]),
        "flb_batch_info": (C.c_int, [H, C.POINTER(C.c_int64)]),
        "flb_batch_set_launch": (C.c_int, [H, C.c_int, C.c_int, C.c_int, C.c_int]),
        "flb_batch_set_wait_limit": (C.c_int, [H, C.c_uint32]),
        "flb_batch_tune": (C.c_int, [H, C.c_uint32, C.c_int]),
        "flb_batch_destroy": (C.c_int, [H]),
        "flb_batch_last_error": (C.c_char_p, [H]),
        "flb_adjoint_desc_init": (None, [C.POINTER(AdjointDesc)]),
        "flb_adjoint_create": (C.c_int, [C.POINTER(AdjointDesc), C.POINTER(H)]),
        "flb_adjoint_set_porosity": (C.c_int, [H, C.c_void_p]),
        "flb_adjoint_set_force": (C.c_int, [H, C.c_double, C.c_double]),
        "flb_adjoint_forward": (C.c_int, [H, C.POINTER(C.c_double)]),
        "flb_adjoint_backward": (C.c_int, [H, C.c_void_p, C.c_void_p]),
        "flb_adjoint_timing": (C.c_int, [H, C.POINTER(C.c_double)]),
        "flb_adjoint_destroy": (C.c_int, [H]),
        "flb_adjoint_last_error": (C.c_char_p, [H]),
        "flb_setup_from_files": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(SetupStruct)]),
        "flb_setup_free": (None, [C.POINTER(SetupStruct)]),
        "flb_setup_initial_flags": (C.c_int, [C.POINTER(SetupStruct), C.c_void_p]),
        "flb_setup_write_mesh_vti": (C.c_int, [C.POINTER(SetupStruct), C.c_char_p]),
        "flb_create_from_files": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(H)]),
        "flb_write_vti": (C.c_int, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.POINTER(VtiField), C.c_uint32]),
        "flb_write_vti_series": (C.c_int, [C.c_char_p, C.c_uint32, C.c_double]),
        "flb_run_from_files": (C.c_int, [C.c_char_p, C.c_char_p, C.c_char_p, C.c_uint64, C.POINTER(RunInfo)]),
        "flb_viz_velocity": (C.c_int, [H, C.c_void_p, C.c_int]),
        "flb_viz_shade": (C.c_int, [H, C.c_int, C.c_void_p, C.c_uint32, C.c_float, C.c_float, C.c_void_p, C.c_int]),
        "flb_viz_isoline": (C.c_int, [H, C.c_int, C.c_float, C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32),
                                      C.c_void_p, C.c_int]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def total_mass_noalloc(mass_ptr: int, excess_ptr: int, flags_ptr: int, nx: int, ny: int, fs_mode: int,
                       out_ptr: int, stream: int = 0):
    """flb_total_mass_noalloc on raw device pointers: enqueues the FP64 free-surface
    mass sum into the device double at ``out_ptr`` on ``stream`` and returns at once."""
    st = load_library().flb_total_mass_noalloc(C.c_void_p(mass_ptr), C.c_void_p(excess_ptr),
                                               C.c_void_p(flags_ptr), int(nx), int(ny), int(fs_mode),
                                               C.c_void_p(out_ptr), C.c_void_p(stream))
    if st != 0:
        raise FlowLBError(st, "flb_total_mass_noalloc")


def _dtype(elem_size: int, field: int):
    if field == FIELD_FLAGS:
        return np.uint8
    return {8: np.float64, 4: np.float32}[elem_size]


class Solver:
    """One case on one GPU.

    Parameters mirror FlowLB's OptionsCalculation (``src/io/reader.h:98-127``):
    ``free_surface`` (TYPE_PROBLEM), ``precision`` (PRECISION 64/32, plus 16 for
    FP16 scaled-deviation storage), ``tau`` (RELAXATION_TIME), ``fx, fy``
    (VOLUMETRIC_FORCE in lattice units), ``collision`` (0 SRT, 1 TRT),
    ``subgrid`` (SUBGRID_TURBULENCE_MODEL).
    """

    def __init__(self, flags: np.ndarray, *, free_surface: bool = False, precision: int = 32,
                 mass_precision: int = 64, tau: float = 0.6, fx: float = 0.0, fy: float = 0.0,
                 use_force: bool = True, collision: int = 0, subgrid: bool = False,
                 bounce_back: int = BB_HALFWAY, fs_mode: int = FS_CONSERVATIVE, inlet_ux: float = 0.0,
                 inlet_uy: float = 0.0, f16_scale: float = 0.0, device: int = -1, stream: int | None = None,
                 kernel_variant: int = 0, u_max: float = 0.0, arithmetic: int = ARITH_FUSED):
        L = load_library()
        g = np.ascontiguousarray(flags, dtype=np.uint8)
        if g.ndim != 2:
            raise ValueError("flags must be a (ny, nx) array")
        self.ny, self.nx = g.shape
        self.N = self.nx * self.ny
        d = CaseDesc()
        L.flb_case_desc_init(C.byref(d))
        d.nx, d.ny, d.flags = self.nx, self.ny, g.ctypes.data
        d.free_surface = int(free_surface)
        d.precision, d.mass_precision = int(precision), int(mass_precision)
        d.collision, d.subgrid, d.use_volumetric_force = int(collision), int(subgrid), int(use_force)
        d.tau, d.fx, d.fy = tau, fx, fy
        d.inlet_ux, d.inlet_uy = inlet_ux, inlet_uy
        d.bounce_back, d.fs_mode, d.f16_scale, d.device = int(bounce_back), int(fs_mode), f16_scale, int(device)
        d.stream = stream or None
        d.kernel_variant = int(kernel_variant)
        d.u_max = float(u_max)
        d.arithmetic = int(arithmetic)
        self._desc = d
        self.free_surface = bool(free_surface)
        self.precision = precision
        h = C.c_void_p()
        st = L.flb_create(C.byref(d), C.byref(h))
        if st != 0:
            raise FlowLBError(st, "flb_create failed")
        self._h = h

    # -- lifetime -------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            load_library().flb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != 0:
            msg = load_library().flb_last_error(self._h)
            raise FlowLBError(st, msg.decode() if msg else "")

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- stepping -----------------------------------------------------------
    def step(self, n: int = 1):
        self._check(load_library().flb_step(self._h, int(n)))

    def sync(self):
        self._check(load_library().flb_sync(self._h))

    def reset(self, flags: np.ndarray):
        g = np.ascontiguousarray(flags, dtype=np.uint8)
        assert g.shape == (self.ny, self.nx)
        self._check(load_library().flb_reset(self._h, g.ctypes.data))

    def run_pass(self, p: int):
        self._check(load_library().flb_run_pass(self._h, int(p)))

    @property
    def t(self) -> int:
        v = C.c_uint64()
        self._check(load_library().flb_get_time(self._h, C.byref(v)))
        return int(v.value)

    @property
    def stream(self) -> int:
        v = C.c_void_p()
        self._check(load_library().flb_get_stream(self._h, C.byref(v)))
        return int(v.value or 0)

    def set_step_mode(self, mode: int):
        """STEP_AUTO, STEP_KERNELS or STEP_PERSISTENT (flb_set_step_mode)."""
        self._check(load_library().flb_set_step_mode(self._h, int(mode)))

    @property
    def persistent(self) -> bool:
        """Whether graph-replayed free-surface steps run as one persistent kernel."""
        m, p = C.c_int(), C.c_int()
        self._check(load_library().flb_get_step_mode(self._h, C.byref(m), C.byref(p)))
        return bool(p.value)

    def set_wait_limit(self, polls: int):
        """Grid-barrier polls of the persistent step before it gives up (0: default)."""
        self._check(load_library().flb_set_wait_limit(self._h, int(polls)))

    def set_stream(self, stream: int | None):
        self._check(load_library().flb_set_stream(self._h, stream or None))

    @property
    def launches(self) -> int:
        v = C.c_uint64()
        self._check(load_library().flb_launch_count(self._h, C.byref(v)))
        return int(v.value)

    # -- fields ---------------------------------------------------------------
    def field_info(self, field: int) -> tuple[int, int]:
        es, n = C.c_size_t(), C.c_size_t()
        self._check(load_library().flb_field_info(self._h, field, C.byref(es), C.byref(n)))
        return int(es.value), int(n.value)

    def read(self, field: int, out: np.ndarray | None = None) -> np.ndarray:
        es, n = self.field_info(field)
        dt = _dtype(es, field)
        if out is None:
            out = np.empty(n, dtype=dt)
        assert out.dtype == dt and out.size == n and out.flags.c_contiguous
        self._check(load_library().flb_read_field(self._h, field, out.ctypes.data, 0))
        return out

    def read_device(self, field: int, dst_ptr: int):
        self._check(load_library().flb_read_field(self._h, field, C.c_void_p(dst_ptr), 1))

    def write(self, field: int, values: np.ndarray):
        es, n = self.field_info(field)
        v = np.ascontiguousarray(values, dtype=_dtype(es, field))
        assert v.size == n
        self._check(load_library().flb_write_field(self._h, field, v.ctypes.data, 0))

    f = property(lambda self: self.read(FIELD_F))
    rho = property(lambda self: self.read(FIELD_RHO))
    u = property(lambda self: self.read(FIELD_U))
    flags = property(lambda self: self.read(FIELD_FLAGS))
    mass = property(lambda self: self.read(FIELD_MASS))
    excess = property(lambda self: self.read(FIELD_EXCESS))
    phi = property(lambda self: self.read(FIELD_PHI))

    def total_mass(self) -> float:
        v = C.c_double()
        self._check(load_library().flb_total_mass(self._h, C.byref(v)))
        return float(v.value)

    def cell_counts(self) -> dict:
        arr = (C.c_uint64 * 4)()
        self._check(load_library().flb_cell_counts(self._h, arr))
        return dict(fluid=int(arr[0]), interface=int(arr[1]), gas=int(arr[2]), wall=int(arr[3]))

    def check_finite(self) -> bool:
        st = load_library().flb_check_finite(self._h)
        if st == 6:
            return False
        self._check(st)
        return True

    def profile_steps(self, n: int) -> dict:
        """Runs n steps with CUDA events around every pass; device ms per pass kind."""
        arr = (C.c_double * 3)()
        self._check(load_library().flb_profile_steps(self._h, int(n), arr))
        return dict(stream_collide=arr[0], fs1=arr[1], fs234=arr[2])

    def profile_phases(self, n: int) -> dict:
        """Runs n steps of the persistent free-surface step with its phases
        timed on the device clock; summed ms per phase (they add up to the
        step time of the production kernel)."""
        arr = (C.c_double * 3)()
        self._check(load_library().flb_profile_phases(self._h, int(n), arr))
        return dict(fs1=arr[0], stream_collide=arr[1], fs234=arr[2])

    def save_checkpoint(self, path: str):
        self._check(load_library().flb_save_checkpoint(self._h, path.encode()))

    def load_checkpoint(self, path: str):
        self._check(load_library().flb_load_checkpoint(self._h, path.encode()))

    # -- headless visualisation ----------------------------------------------
    def viz_velocity(self) -> np.ndarray:
        """(ny, nx, 2) float32: the velocity image of save2DDataToOpenGL."""
        out = np.empty((self.ny, self.nx, 2), np.float32)
        self._check(load_library().flb_viz_velocity(self._h, out.ctypes.data, 0))
        return out

    def viz_shade(self, quantity: int, colormap: np.ndarray, max_value: float, min_value: float) -> np.ndarray:
        """(ny, nx, 4) uint8 RGBA: one shaded pixel per node."""
        cm = np.ascontiguousarray(colormap, np.float32).reshape(-1, 3)
        out = np.empty((self.ny, self.nx, 4), np.uint8)
        self._check(load_library().flb_viz_shade(self._h, int(quantity), cm.ctypes.data, cm.shape[0],
                                                 float(max_value), float(min_value), out.ctypes.data, 0))
        return out

    def viz_isoline(self, field: int, iso_value: float, width: int, height: int, bounds=None) -> np.ndarray:
        """(height, width) uint8 image of the iso-line (255 on the line)."""
        b = (C.c_uint32 * 4)(*(bounds if bounds is not None else (0, self.nx, 0, self.ny)))
        out = np.empty((height, width), np.uint8)
        self._check(load_library().flb_viz_isoline(self._h, int(field), float(iso_value), int(width), int(height), b,
                                                   out.ctypes.data, 0))
        return out

    @classmethod
    def from_files(cls, geometry_txt: str, options_txt: str) -> "Solver":
        """``flb_create_from_files``: the case FlowLB's ``App::calculate`` would
        run from these two files, in the reference's modes."""
        L = load_library()
        st_setup = Setup(geometry_txt, options_txt)  # raises with the reader's message
        h = C.c_void_p()
        st = L.flb_create_from_files(geometry_txt.encode(), options_txt.encode(), C.byref(h))
        if st != 0:
            raise FlowLBError(st, "flb_create_from_files failed")
        self = cls.__new__(cls)
        self._h = h
        self.nx, self.ny, self.N = st_setup.nx, st_setup.ny, st_setup.nx * st_setup.ny
        self._desc = st_setup.desc
        self.free_surface = bool(st_setup.desc.free_surface)
        self.precision = int(st_setup.desc.precision)
        return self


class Setup:
    """``flb_setup_from_files``: Geometry.txt + OptionsCalc.txt to geometry
    flags, tau, force, inlet velocity and loop bounds (host only, no GPU)."""

    def __init__(self, geometry_txt: str, options_txt: str, mesh_only: bool = False):
        L = load_library()
        s = SetupStruct()
        st = L.flb_setup_from_files(geometry_txt.encode(), options_txt.encode(), int(mesh_only), C.byref(s))
        if st != 0:
            raise FlowLBError(st, s.error.decode(errors="replace"))
        try:
            self.nx, self.ny = int(s.nx), int(s.ny)
            self.flags = np.ctypeslib.as_array(C.cast(s.flags, C.POINTER(C.c_uint8)), (self.ny, self.nx)).copy()
            init = np.empty((self.ny, self.nx), np.uint8)
            st = L.flb_setup_initial_flags(C.byref(s), init.ctypes.data)
            if st != 0:
                raise FlowLBError(st, "flb_setup_initial_flags failed")
            self.initial_flags = init
            self.origin = (s.x_min, s.y_min, s.z_min)
            self.spacing = s.spacing
            d = CaseDesc()
            C.memmove(C.byref(d), C.byref(s.desc), C.sizeof(CaseDesc))
            d.flags = None
            self.desc = d
            self.time_steps, self.save_every = int(s.time_steps), int(s.save_every)
            self.time_simulation, self.time_save = float(s.time_simulation), float(s.time_save)
            self.nu_lattice = float(s.nu_lattice)
            self.units = dict(length=s.length_to_si, time=s.time_to_si, mass=s.mass_to_si,
                              velocity=s.velocity_to_si, rho=s.rho_to_si)
            self.graphics_api, self.reference_precision = int(s.graphics_api), int(s.reference_precision)
            self.cuda_block = tuple(int(v) for v in s.cuda_block)
        finally:
            L.flb_setup_free(C.byref(s))

    def write_mesh_vti(self, path: str):
        """App::createDomain's mesh.vti for these flags."""
        write_vti(path, [("Flags", self.initial_flags.ravel(), 1, 1.0, False)], self.nx, self.ny,
                  self.origin, self.spacing)


def write_vti(path: str, fields, nx: int, ny: int, origin=(0.0, 0.0, 0.0), spacing: float = 1.0):
    """``flb_write_vti``.  ``fields``: (name, array, components, to_si, flip_y)
    with arrays of uint8, float32 or float64 holding components x N values."""
    L = load_library()
    keep = []
    arr = (VtiField * max(1, len(fields)))()
    kinds = {np.dtype(np.uint8): VTI_UINT8, np.dtype(np.float32): VTI_FLOAT32, np.dtype(np.float64): VTI_FLOAT64}
    for k, (name, data, comps, to_si, flip) in enumerate(fields):
        a = np.ascontiguousarray(data)
        if a.dtype not in kinds or a.size != comps * nx * ny:
            raise ValueError(f"field {name}: need {comps}*{nx}*{ny} values of uint8/float32/float64")
        nm = name.encode()
        keep += [a, nm]
        arr[k] = VtiField(nm, kinds[a.dtype], int(comps), a.ctypes.data, float(to_si), int(bool(flip)))
    st = L.flb_write_vti(path.encode(), nx, ny, float(origin[0]), float(origin[1]), float(origin[2]),
                         float(spacing), arr, len(fields))
    if st != 0:
        raise FlowLBError(st, f"flb_write_vti({path}) failed")


def run_from_files(geometry_txt: str, options_txt: str, save_dir: str, max_steps: int = 0) -> dict:
    """``flb_run_from_files``: FlowLB's headless run from its two input files."""
    L = load_library()
    info = RunInfo()
    st = L.flb_run_from_files(geometry_txt.encode(), options_txt.encode(), save_dir.encode(), int(max_steps),
                              C.byref(info))
    if st != 0:
        raise FlowLBError(st, info.error.decode(errors="replace"))
    return dict(steps=int(info.steps), files=int(info.files), directory=info.directory.decode())


class Batch:
    """Many independent single-phase FP32 cases advanced by one persistent
    kernel per ``step`` call (``flb_batch_*``).  ``cases``: a list of
    ``(flags, tau, fx, fy)``; the wall treatment and arithmetic are shared.
    ``autotune``: 0 fixed launch shape, 1 timed search at creation (or a probe
    step count > 1)."""

    def __init__(self, cases, *, bounce_back: int = BB_HALFWAY, arithmetic: int = ARITH_FUSED, autotune: int = 1,
                 device: int = -1, stream: int | None = None):
        L = load_library()
        self._flags = [np.ascontiguousarray(c[0], dtype=np.uint8) for c in cases]
        n = len(self._flags)
        descs = (CaseDesc * n)()
        self.shapes = []
        for i, (g, c) in enumerate(zip(self._flags, cases)):
            d = descs[i]
            L.flb_case_desc_init(C.byref(d))
            ny, nx = g.shape
            self.shapes.append((ny, nx))
            d.nx, d.ny, d.flags = nx, ny, g.ctypes.data
            d.precision = 32
            d.tau, d.fx, d.fy = float(c[1]), float(c[2]), float(c[3])
            d.bounce_back, d.arithmetic, d.device = int(bounce_back), int(arithmetic), int(device)
            d.stream = stream or None
        h = C.c_void_p()
        st = L.flb_batch_create(descs, n, int(autotune), C.byref(h))
        if st != 0:
            raise FlowLBError(st, "flb_batch_create failed")
        self._h = h
        self.n = n

    def _check(self, st: int):
        if st != 0:
            msg = load_library().flb_batch_last_error(self._h)
            raise FlowLBError(st, msg.decode() if msg else "")

    def step(self, n: int = 1):
        self._check(load_library().flb_batch_step(self._h, int(n)))

    def sync(self):
        self._check(load_library().flb_batch_sync(self._h))

    def reset(self):
        self._check(load_library().flb_batch_reset(self._h))

    def info(self) -> dict:
        a = (C.c_int64 * 8)()
        self._check(load_library().flb_batch_info(self._h, a))
        mode = "streams" if a[7] == BATCH_STREAMS else "team" if (a[7] & ~BATCH_VECTOR) == BATCH_TEAM else "cluster"
        return dict(cases=a[0], cells=a[1], t=a[2], group=a[3], groups=a[4], tuned=bool(a[5]), threads=a[6],
                    mode=mode, vector=bool(a[7] & BATCH_VECTOR) and mode != "streams")

    def set_launch(self, mode: str, group: int, groups: int, threads: int, vector: bool = False):
        """Launch shape for the following steps: ``mode`` "cluster" or "team",
        CTAs per group, groups, threads per CTA (``info()`` of a tuned batch,
        for instance), and the vector data path; or "streams" with group 1
        and ``groups`` streams (each case its own handle, the cases' step
        graphs on concurrent streams; an even step only).  The state is kept."""
        m = ({"cluster": BATCH_CLUSTER, "team": BATCH_TEAM, "streams": BATCH_STREAMS}[mode]
             | (BATCH_VECTOR if vector else 0))
        self._check(load_library().flb_batch_set_launch(self._h, m, int(group), int(groups), int(threads)))

    def tune(self, probe_steps: int = 0, forms: int = TUNE_PERSISTENT | TUNE_STREAMS):
        """Times the launch shapes of the given forms again, keeps the fastest
        and restarts from the initial state (t = 0)."""
        self._check(load_library().flb_batch_tune(self._h, int(probe_steps), int(forms)))

    def set_wait_limit(self, polls: int):
        """Polls a team-mode CTA waits at its team's barrier before the launch
        gives up (0: the default, 2^21)."""
        self._check(load_library().flb_batch_set_wait_limit(self._h, int(polls)))

    def read(self, i: int, field: int) -> np.ndarray:
        ny, nx = self.shapes[i]
        N = nx * ny
        count = {FIELD_F: 9 * N, FIELD_RHO: N, FIELD_U: 2 * N, FIELD_FLAGS: N}[field]
        out = np.empty(count, dtype=np.uint8 if field == FIELD_FLAGS else np.float32)
        self._check(load_library().flb_batch_read_field(self._h, int(i), field, out.ctypes.data, 0))
        return out

    def close(self):
        if getattr(self, "_h", None):
            load_library().flb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """Forward/backward pair of the Brinkman-porosity single phase
    (``flb_adjoint_*``): ``forward()`` returns J, ``backward()`` returns
    (dJ/ds as (ny, nx), dJ/dg as (2,))."""

    def __init__(self, flags: np.ndarray, porosity: np.ndarray, *, tau: float = 0.6, gx: float = 0.0,
                 gy: float = 0.0, precision: int = 32, steps: int = 4096, window: int = 512,
                 checkpoint_every: int = 64, device: int = -1, stream: int | None = None):
        L = load_library()
        self._flags = np.ascontiguousarray(flags, dtype=np.uint8)
        s = np.ascontiguousarray(porosity, dtype=np.float64)
        self.ny, self.nx = self._flags.shape
        d = AdjointDesc()
        L.flb_adjoint_desc_init(C.byref(d))
        d.nx, d.ny, d.flags, d.porosity = self.nx, self.ny, self._flags.ctypes.data, s.ctypes.data
        d.precision, d.tau, d.gx, d.gy = int(precision), float(tau), float(gx), float(gy)
        d.steps, d.window, d.checkpoint_every = int(steps), int(window), int(checkpoint_every)
        d.device, d.stream = int(device), stream or None
        h = C.c_void_p()
        st = L.flb_adjoint_create(C.byref(d), C.byref(h))
        if st != 0:
            raise FlowLBError(st, "flb_adjoint_create failed")
        self._h = h

    def _check(self, st: int):
        if st != 0:
            msg = load_library().flb_adjoint_last_error(self._h)
            raise FlowLBError(st, msg.decode() if msg else "")

    def set_porosity(self, porosity: np.ndarray):
        s = np.ascontiguousarray(porosity, dtype=np.float64)
        assert s.size == self.nx * self.ny
        self._check(load_library().flb_adjoint_set_porosity(self._h, s.ctypes.data))

    def set_force(self, gx: float, gy: float = 0.0):
        self._check(load_library().flb_adjoint_set_force(self._h, float(gx), float(gy)))

    def forward(self) -> float:
        J = C.c_double()
        self._check(load_library().flb_adjoint_forward(self._h, C.byref(J)))
        return float(J.value)

    def backward(self):
        ds = np.empty(self.nx * self.ny)
        dg = np.empty(2)
        self._check(load_library().flb_adjoint_backward(self._h, ds.ctypes.data, dg.ctypes.data))
        return ds.reshape(self.ny, self.nx), dg

    def timing(self) -> tuple[float, float]:
        a = (C.c_double * 2)()
        self._check(load_library().flb_adjoint_timing(self._h, a))
        return float(a[0]), float(a[1])

    def close(self):
        if getattr(self, "_h", None):
            load_library().flb_adjoint_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
