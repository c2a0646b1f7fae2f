"""ctypes front end of the CPU oracle and of the reference's own libraries.

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()``
as the checker, and by the CPU-baseline leg of ``bench.py``.  The engine in
``flowlb_b200`` never imports it.

* ``Oracle``: the C restatement of the reference step (``liboracle.so``).
* ``ref_host_init``: the reference's own host initialisation
  (``_ref/libflbref_host.so``, built from FlowLB ``src/initData.cpp``).
* ``ref_cuda_run`` / ``ref_cuda_time``: the reference's own CUDA kernels
  (``_ref/libflbref_cuda.so``, built from FlowLB ``src/cuda/*.cu`` with
  ``--fmad=false``); needs a GPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

F64, F32, F16S, F32_M32 = 0, 1, 2, 3
BB_IMPLICIT, BB_HALFWAY = 0, 1
FS_REFERENCE, FS_CONSERVATIVE = 0, 1
ARITH_REFERENCE, ARITH_FUSED = 0, 1
K_STREAM_COLLIDE, K_FS1, K_FS2, K_FS3, K_FS4 = 0, 1, 2, 3, 4
FIELD_F, FIELD_RHO, FIELD_U, FIELD_FLAGS, FIELD_MASS, FIELD_EXCESS, FIELD_PHI = range(7)


class OrcParams(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("variant", C.c_int32), ("free_surface", C.c_int32),
        ("bb", C.c_int32), ("fs_mode", C.c_int32), ("collision", C.c_int32), ("subgrid", C.c_int32),
        ("use_force", C.c_int32), ("fs_count_pre", C.c_int32), ("fs1_post", C.c_int32), ("tau", C.c_float),
        ("fx", C.c_float),
        ("fy", C.c_float), ("f16_scale", C.c_float), ("threads", C.c_int32), ("inlet_ux", C.c_double),
        ("inlet_uy", C.c_double), ("u_max", C.c_float), ("arithmetic", C.c_int32),
    ]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle`")
        L = C.CDLL(path)
        L.orc_adj_run.restype = C.c_int
        L.orc_adj_run.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                  C.c_double, C.c_uint64, C.c_uint64, C.POINTER(C.c_double), C.c_void_p,
                                  C.c_void_p]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_void_p]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_uint64]
        L.orc_kernel.argtypes = [C.c_void_p, C.c_int]
        L.orc_time.restype = C.c_uint64
        L.orc_time.argtypes = [C.c_void_p]
        L.orc_set_time.argtypes = [C.c_void_p, C.c_uint64]
        L.orc_cells.restype = C.c_size_t
        L.orc_cells.argtypes = [C.c_void_p]
        L.orc_field.restype = C.c_void_p
        L.orc_field.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
        L.orc_read_f64.argtypes = [C.c_void_p, C.c_void_p]
        L.orc_total_mass.restype = C.c_double
        L.orc_total_mass.argtypes = [C.c_void_p]
        L.orc_f16_rs_pair.restype = C.c_uint32
        L.orc_f16_rs_pair.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        L.orc_fs1_options.restype = C.c_int
        L.orc_fs1_options.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p, C.c_void_p]
        L.orc_fs4_options.restype = C.c_int
        L.orc_fs4_options.argtypes = [C.c_void_p, C.c_size_t, C.c_void_p]
        _lib = L
    return _lib


def _ctype(variant: int, field: int):
    if field == FIELD_FLAGS:
        return np.uint8
    if field == FIELD_F:
        return {F64: np.float64, F32: np.float32, F16S: np.float16, F32_M32: np.float32}[variant]
    if field in (FIELD_RHO, FIELD_U):
        return np.float64 if variant == F64 else np.float32
    return np.float32 if variant == F32_M32 else np.float64


@dataclass
class OracleConfig:
    variant: int = F32
    free_surface: bool = False
    bb: int = BB_IMPLICIT
    fs_mode: int = FS_REFERENCE
    collision: int = 0
    subgrid: bool = False
    use_force: bool = True
    fs_count_pre: bool = False
    fs1_post: bool = False
    tau: float = 0.6
    fx: float = 0.0
    fy: float = 0.0
    inlet_ux: float = 0.0
    inlet_uy: float = 0.0
    f16_scale: float = 4096.0
    threads: int = 0
    u_max: float = 0.0
    arithmetic: int = ARITH_REFERENCE


class Oracle:
    """One case on the CPU oracle.  Field accessors return numpy views of the
    oracle's own arrays (writable: tests plant states through them)."""

    def __init__(self, geometry_flags: np.ndarray, cfg: OracleConfig):
        g = np.ascontiguousarray(geometry_flags, dtype=np.uint8)
        self.ny, self.nx = g.shape
        self.N = self.nx * self.ny
        self.cfg = cfg
        p = OrcParams(self.nx, self.ny, cfg.variant, int(cfg.free_surface), cfg.bb, cfg.fs_mode, cfg.collision,
                      int(cfg.subgrid), int(cfg.use_force), int(cfg.fs_count_pre), int(cfg.fs1_post), cfg.tau,
                      cfg.fx, cfg.fy,
                      cfg.f16_scale, cfg.threads, cfg.inlet_ux, cfg.inlet_uy, cfg.u_max, cfg.arithmetic)
        self._h = lib().orc_create(C.byref(p), g.ctypes.data)
        if not self._h:
            raise ValueError("orc_create rejected the case")

    def close(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    @property
    def t(self) -> int:
        return int(lib().orc_time(self._h))

    @t.setter
    def t(self, value: int):
        lib().orc_set_time(self._h, int(value))

    def step(self, n: int = 1):
        lib().orc_step(self._h, int(n))

    def kernel(self, k: int):
        if lib().orc_kernel(self._h, int(k)) != 0:
            raise ValueError(f"kernel {k} not available in this mode")

    def field(self, which: int) -> np.ndarray:
        es = C.c_size_t()
        ptr = lib().orc_field(self._h, which, C.byref(es))
        count = {FIELD_F: 9 * self.N, FIELD_U: 2 * self.N}.get(which, self.N)
        dt = np.dtype(_ctype(self.cfg.variant, which))
        assert dt.itemsize == es.value
        buf = (C.c_char * (count * dt.itemsize)).from_address(ptr)
        return np.frombuffer(buf, dtype=dt, count=count)

    f = property(lambda self: self.field(FIELD_F))
    rho = property(lambda self: self.field(FIELD_RHO))
    u = property(lambda self: self.field(FIELD_U))
    flags = property(lambda self: self.field(FIELD_FLAGS))
    mass = property(lambda self: self.field(FIELD_MASS))
    excess = property(lambda self: self.field(FIELD_EXCESS))
    phi = property(lambda self: self.field(FIELD_PHI))

    def f64(self) -> np.ndarray:
        out = np.empty(9 * self.N, dtype=np.float64)
        lib().orc_read_f64(self._h, out.ctypes.data)
        return out

    def total_mass(self) -> float:
        return float(lib().orc_total_mass(self._h))

    def fs1_options(self, idx: int):
        """Every result the reference FS_1 kernel can give for cell idx (state
        before FS_1): list of (mass, rebuilt[8], mask)."""
        m = np.zeros(256)
        r = np.zeros(256 * 8)
        k = np.zeros(256, np.uint8)
        n = lib().orc_fs1_options(self._h, int(idx), m.ctypes.data, r.ctypes.data, k.ctypes.data)
        return [(m[c], r[8 * c:8 * c + 8], int(k[c])) for c in range(max(n, 0))]

    def fs4_options(self, idx: int):
        """Every (mass, excess, fill level) the reference FS_4 kernel can give
        for cell idx (state after FS_3)."""
        out = np.zeros(27)
        n = lib().orc_fs4_options(self._h, int(idx), out.ctypes.data)
        return [tuple(out[3 * c:3 * c + 3]) for c in range(max(n, 0))]


# ---- the reference's own code ---------------------------------------------
REF_DIR = os.path.join(HERE, "_ref")


def ref_host_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libflbref_host.so"))


def ref_cuda_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libflbref_cuda.so"))


def ref_host_init(geometry_flags: np.ndarray, precision: int, free_surface: bool,
                  inlet_ux: float = 0.0, inlet_uy: float = 0.0) -> dict:
    """Initial state built by FlowLB's own initFields / initFreeSurfaceFlags /
    initFreeSurfaceFields."""
    L = C.CDLL(os.path.join(REF_DIR, "libflbref_host.so"))
    L.ref_host_init.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_double, C.c_double] + \
        [C.c_void_p] * 7
    g = np.ascontiguousarray(geometry_flags, dtype=np.uint8)
    ny, nx = g.shape
    N = nx * ny
    dt = np.float32 if precision == 32 else np.float64
    out = dict(f=np.zeros(9 * N, dt), u=np.zeros(2 * N, dt), rho=np.zeros(N, dt), flags=np.zeros(N, np.uint8),
               phi=np.zeros(N, dt), mass=np.zeros(N, dt), excess=np.zeros(N, dt))
    rc = L.ref_host_init(precision, nx, ny, g.ctypes.data, int(free_surface), inlet_ux, inlet_uy,
                         out["f"].ctypes.data, out["u"].ctypes.data, out["rho"].ctypes.data,
                         out["flags"].ctypes.data, out["phi"].ctypes.data, out["mass"].ctypes.data,
                         out["excess"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_host_init failed: {rc}")
    return out


def ref_cuda_run(state: dict, nx: int, ny: int, precision: int, free_surface: bool, tau: float, fx: float,
                 fy: float, t0: int, nsteps: int = 0, kernel_id: int = -1, collision: int = 0,
                 subgrid: bool = False, use_force: bool = True) -> dict:
    """Runs the reference CUDA kernels on a copy of ``state`` (keys f, rho, u,
    flags, mass, excess, phi in the reference layout) and returns the result."""
    L = C.CDLL(os.path.join(REF_DIR, "libflbref_cuda.so"))
    L.ref_cuda_run.argtypes = [C.c_int] * 7 + [C.c_double] * 3 + [C.c_uint64, C.c_uint64, C.c_int] + \
        [C.c_void_p] * 7
    dt = np.float32 if precision == 32 else np.float64
    s = {k: np.ascontiguousarray(np.array(v, copy=True), dtype=(np.uint8 if k == "flags" else dt))
         for k, v in state.items()}
    N = nx * ny
    for k in ("mass", "excess", "phi"):
        if k not in s:
            s[k] = np.zeros(N, dt)
    rc = L.ref_cuda_run(precision, nx, ny, int(free_surface), collision, int(subgrid), int(use_force),
                        float(tau), float(fx), float(fy), int(t0), int(nsteps), int(kernel_id),
                        s["f"].ctypes.data, s["rho"].ctypes.data, s["u"].ctypes.data, s["flags"].ctypes.data,
                        s["mass"].ctypes.data, s["excess"].ctypes.data, s["phi"].ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_cuda_run failed: {rc}")
    return s


def ref_cuda_timing_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libflbref_cuda_timing.so"))


def ref_cuda_time(state: dict, nx: int, ny: int, precision: int, free_surface: bool, tau: float, fx: float,
                  fy: float, warm: int, nsteps: int, t0: int = 0, build: str = "parity") -> tuple:
    """Device time of the reference's own CUDA step sequence (16x16 blocks, one
    launch per kernel and step, as its headless loop issues them): ``warm``
    untimed steps from ``state`` at ``t0``, then ``nsteps`` timed with CUDA
    events.  ``build``: "parity" (the kernels as written, no floating-point
    contraction: bit-comparable) or "timing" (FlowLB's own build flags with
    the debug printf calls compiled out).  Returns (milliseconds, final state)."""
    lib_name = {"parity": "libflbref_cuda.so", "timing": "libflbref_cuda_timing.so"}[build]
    L = C.CDLL(os.path.join(REF_DIR, lib_name))
    L.ref_cuda_time.argtypes = [C.c_int] * 7 + [C.c_double] * 3 + [C.c_uint64] * 3 + [C.c_void_p] * 8
    dt = np.float32 if precision == 32 else np.float64
    s = {k: np.ascontiguousarray(np.array(v, copy=True), dtype=(np.uint8 if k == "flags" else dt))
         for k, v in state.items()}
    N = nx * ny
    for k in ("mass", "excess", "phi"):
        if k not in s:
            s[k] = np.zeros(N, dt)
    ms = C.c_double()
    rc = L.ref_cuda_time(precision, nx, ny, int(free_surface), 0, 0, 1, float(tau), float(fx), float(fy), int(t0),
                         int(warm), int(nsteps), s["f"].ctypes.data, s["rho"].ctypes.data, s["u"].ctypes.data,
                         s["flags"].ctypes.data, s["mass"].ctypes.data, s["excess"].ctypes.data,
                         s["phi"].ctypes.data, C.byref(ms))
    if rc != 0:
        raise RuntimeError(f"ref_cuda_time failed: {rc}")
    return float(ms.value), s


def ref_cuda_isoline(field: np.ndarray, nx: int, ny: int, precision: int, iso: float, width: int, height: int,
                     bounds) -> np.ndarray:
    """The reference's own iso-line kernel (d_CreateIsoSurfaceVector2D) on a
    two-component field (2N values, reference layout) into a (height, width)
    uint8 image.  Only camera bounds inside the lattice and finite values are
    accepted (the kernel writes through a surface that traps out of range)."""
    L = C.CDLL(os.path.join(REF_DIR, "libflbref_cuda.so"))
    L.ref_cuda_isoline.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_float, C.c_uint, C.c_uint,
                                   C.POINTER(C.c_uint), C.c_void_p]
    dt = np.float32 if precision == 32 else np.float64
    v = np.ascontiguousarray(field, dtype=dt)
    assert v.size == 2 * nx * ny
    b = (C.c_uint * 4)(*[int(k) for k in bounds])
    img = np.zeros((height, width), np.uint8)
    rc = L.ref_cuda_isoline(precision, nx, ny, v.ctypes.data, float(iso), width, height, b, img.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"ref_cuda_isoline failed: {rc}")
    return img


def adjoint_run(flags: np.ndarray, porosity: np.ndarray, tau: float, gx: float, gy: float, steps: int,
                window: int, grad: bool = True):
    """FP64 CPU tape adjoint of the Brinkman-porosity step (flb_adjoint_oracle.c):
    returns (J, dJ/ds as (ny, nx), dJ/dg as (2,)) or (J, None, None)."""
    g = np.ascontiguousarray(flags, dtype=np.uint8)
    sv = np.ascontiguousarray(porosity, dtype=np.float64)
    ny, nx = g.shape
    J = C.c_double()
    ds = np.zeros(nx * ny) if grad else None
    dg = np.zeros(2) if grad else None
    rc = lib().orc_adj_run(nx, ny, g.ctypes.data, sv.ctypes.data, tau, gx, gy, steps, window, C.byref(J),
                           ds.ctypes.data if grad else None, dg.ctypes.data if grad else None)
    if rc != 0:
        raise MemoryError("orc_adj_run")
    return float(J.value), (ds.reshape(ny, nx) if grad else None), dg
