"""Geometry-flag builders for the synthetic culvert cases.

Cell flags use FlowLB's uint8 cell-type encoding (``src/utils.h:91-108``,
``src/cuda/cudaInitData.cu:25-39``).  The builders return the *geometry* flags,
i.e. what FlowLB's geometry stage hands to ``initData`` (``src/initData.h:220-333``):
FLUID / GAS / WALL cells, before the free-surface interface layer is added.
Arrays are ``(ny, nx)`` C-ordered so that ``flags.ravel()[x + y*nx]`` is cell
``(x, y)`` exactly as the reference indexes it.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

FLUID = 0x01
GAS = 0x02
INTERFACE = 0x04
WALL = 0x08
MOVING_WALL = 0x10
INLET = 0x20
OUTLET = 0x40
GAS_INTERFACE = 0x80
INTERFACE_FLUID = INTERFACE | FLUID
INTERFACE_GAS = INTERFACE | GAS


@dataclass
class Case:
    """A synthetic case: geometry flags plus the physical parameters."""

    name: str
    flags: np.ndarray  # (ny, nx) uint8 geometry flags
    tau: float
    fx: float
    fy: float
    free_surface: bool
    steps: int
    porosity: np.ndarray | None = None  # (ny, nx) float32 Brinkman solid fraction
    extra: dict = field(default_factory=dict)

    @property
    def nx(self) -> int:
        return int(self.flags.shape[1])

    @property
    def ny(self) -> int:
        return int(self.flags.shape[0])

    @property
    def cells(self) -> int:
        return self.nx * self.ny


def channel_with_block(nx: int, ny: int, bx0: int, bx1: int, by1: int) -> np.ndarray:
    """Periodic-x channel: wall rows y=0 and y=ny-1, solid block
    x in [bx0, bx1), y in [1, by1) sitting on the bottom wall, fluid elsewhere."""
    flags = np.full((ny, nx), FLUID, dtype=np.uint8)
    flags[0, :] = WALL
    flags[ny - 1, :] = WALL
    flags[1:by1, bx0:bx1] = WALL
    return flags


def plain_channel(nx: int = 256, ny: int = 64, steps: int = 10_000) -> Case:
    """Single-phase culvert channel: 256x64, periodic in x, walls top and
    bottom, 32x24 block centred at x=128 on the bottom wall, g_x=1e-6, tau=0.6."""
    bw = max(2, (32 * nx) // 256)
    bh = max(1, (24 * ny) // 64)
    x0 = nx // 2 - bw // 2
    flags = channel_with_block(nx, ny, x0, x0 + bw, 1 + bh)
    return Case("plain-channel", flags, tau=0.6, fx=1e-6, fy=0.0, free_surface=False, steps=steps)


def dam_break(scale: int = 1, steps: int = 20_000) -> Case:
    """Free-surface culvert dam break.  scale=1: 2048x512; scale=4: 8192x2048.

    Wall frame; water column x < 40% of the width, y < 0.6 H (x from 1, y
    from 1); gas elsewhere; a solid culvert box 256*scale wide and 160*scale
    high, centred at x=1200*scale on the bottom wall, whose lowest 96*scale
    rows are an open barrel through the full length of the box.
    tau=0.55, g_y=-5e-5.
    """
    nx, ny = 2048 * scale, 512 * scale
    flags = np.full((ny, nx), GAS, dtype=np.uint8)
    flags[0, :] = WALL
    flags[ny - 1, :] = WALL
    flags[:, 0] = WALL
    flags[:, nx - 1] = WALL
    col_x = int(np.ceil(0.4 * nx))      # 819 at scale 1, 3277 at scale 4
    col_y = int(np.ceil(0.6 * ny))      # 307 at scale 1, 1229 at scale 4
    flags[1:col_y, 1:col_x] = FLUID
    bw, bh, opening = 256 * scale, 160 * scale, 96 * scale
    cx = 1200 * scale
    bx0, bx1 = cx - bw // 2, cx + bw // 2
    flags[1 + opening:1 + bh, bx0:bx1] = WALL
    return Case(f"dam-break-{nx}x{ny}", flags, tau=0.55, fx=0.0, fy=-5e-5, free_surface=True, steps=steps)


def hbm_probe(nx: int = 8192, ny: int = 2048, steps: int = 2000) -> Case:
    """Single-phase probe on a grid far larger than L2 with the plain-channel physics."""
    c = plain_channel(nx, ny, steps)
    c.name = f"single-phase-{nx}x{ny}"
    return c


def small_dam_break(nx: int = 64, ny: int = 48, steps: int = 200) -> Case:
    """Dam break shrunk to a few thousand cells, for cell-by-cell parity."""
    flags = np.full((ny, nx), GAS, dtype=np.uint8)
    flags[0, :] = WALL
    flags[ny - 1, :] = WALL
    flags[:, 0] = WALL
    flags[:, nx - 1] = WALL
    col_x = int(np.ceil(0.4 * nx))
    col_y = int(np.ceil(0.6 * ny))
    flags[1:col_y, 1:col_x] = FLUID
    bw, bh, opening = max(4, nx // 8), max(3, ny // 3), max(2, ny // 5)
    cx = int(0.6 * nx)
    flags[1 + opening:1 + bh, cx - bw // 2:cx + bw // 2] = WALL
    return Case(f"dam-break-{nx}x{ny}", flags, tau=0.55, fx=0.0, fy=-5e-5, free_surface=True, steps=steps)


ENSEMBLE_SEED = 20261203


def ensemble(n_cases: int = 512, seed: int = ENSEMBLE_SEED, steps: int = 5000) -> list[Case]:
    """Batched culvert ensemble: seed-drawn single-phase channel cases.

    Per case, in this order: nx ~ U[128,1024], ny ~ U[64,256] (integers),
    block width ~ U[0.05,0.2]*nx, block height ~ U[0.2,0.6]*ny, tau ~
    U[0.52,0.8], g_x ~ logU[1e-7,1e-5].  numpy PCG64 generator.
    """
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_cases):
        nx = int(rng.integers(128, 1025))
        ny = int(rng.integers(64, 257))
        w = max(1, int(round(rng.uniform(0.05, 0.2) * nx)))
        h = max(1, int(round(rng.uniform(0.2, 0.6) * ny)))
        tau = float(np.float32(rng.uniform(0.52, 0.8)))
        gx = float(np.float32(10.0 ** rng.uniform(-7.0, -5.0)))
        x0 = nx // 2 - w // 2
        flags = channel_with_block(nx, ny, x0, x0 + w, min(ny - 2, 1 + h))
        out.append(Case(f"ensemble-{k}", flags, tau=tau, fx=gx, fy=0.0, free_surface=False, steps=steps))
    return out


def porous_channel(nx: int = 1024, ny: int = 256, seed: int = 7, steps: int = 4096) -> Case:
    """Adjoint case: periodic-x channel with walls top/bottom and a Brinkman
    solid fraction s in [0,1]: 0.5 + 0.5 * (sum of 8 seeded Fourier modes with
    wavenumbers <= 4, normalised to +-1), clamped, and s = 1 inside the
    culvert block x in [448,576), y in [1,97) (scaled with the grid)."""
    rng = np.random.default_rng(seed)
    flags = np.full((ny, nx), FLUID, dtype=np.uint8)
    flags[0, :] = WALL
    flags[ny - 1, :] = WALL
    yy, xx = np.meshgrid(np.arange(ny) / ny, np.arange(nx) / nx, indexing="ij")
    field_ = np.zeros((ny, nx))
    for _ in range(8):
        kx, ky = rng.integers(0, 5, size=2)
        ph = rng.uniform(0, 2 * np.pi)
        amp = rng.uniform(0.5, 1.0)
        field_ += amp * np.cos(2 * np.pi * (kx * xx + ky * yy) + ph)
    field_ /= max(1e-12, np.abs(field_).max())
    s = np.clip(0.5 + 0.5 * field_, 0.0, 1.0)
    bx0, bx1 = (448 * nx) // 1024, (576 * nx) // 1024
    by1 = 1 + (96 * ny) // 256
    s[1:by1, bx0:bx1] = 1.0
    s[flags == WALL] = 0.0
    return Case("porous-channel", flags, tau=0.6, fx=5e-6, fy=0.0, free_surface=False, steps=steps,
                porosity=s.astype(np.float32))
