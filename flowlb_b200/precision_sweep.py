"""Storage-precision sweep of the free-surface dam break.

The same case is run with the populations stored in FP64, FP32 and FP16
scaled deviations (FP32 arithmetic; mass, excess and fill level in FP64 in
every run), and the FP32 and FP16S results are compared with the FP64 run:

  velocity_l2    ||u - u64|| / ||u64|| over the cells that are fluid or
                 interface in both runs (both velocity components)
  surface_error  mean over the columns of |h - h64|, h(x) the height of the
                 topmost phi = 0.5 crossing of column x (linear
                 interpolation between the cells around it; 0 for a dry
                 column), in cells
  depth_error    mean over the columns of |d - d64|, d(x) = sum over y of phi
                 (the water depth of the column, in cells)
  mass_drift     (M(T) - M(0)) / M(0) of each run's own total mass
                 (flb_total_mass, FP64)

The three runs are stepped side by side and compared at checkpoints
(500 .. 50,000 steps): the dam-break surge is chaotic, so any rounding
difference grows until the trajectories decorrelate, and the series shows
when that happens for FP32 and FP16S alike.

FlowLB parses PRECISION = 16 (src/io/reader.cpp:367) but has no FP16 path
(src/ui/app.cpp:286-316 dispatches float and double only), so the FP64 run
is the reference here; the FP64 engine equals the FP64 CPU oracle bit for
bit on the cases the tests compare.

    python -m flowlb_b200.precision_sweep --scale 4 --steps 50000
"""
from __future__ import annotations

import argparse
import json

import numpy as np

from . import cases
from . import engine as E

LIVE = (cases.FLUID, cases.INTERFACE)


def surface_heights(phi: np.ndarray, flags: np.ndarray) -> np.ndarray:
    """Per column, the height (in cells, cell centres at y + 0.5) of the
    topmost place where the fill level crosses 0.5 going up; 0 for a column
    with no cell at or above 0.5.  Solid cells count as empty."""
    ny, nx = phi.shape
    p = np.where((flags & cases.WALL) != 0, 0.0, phi)
    wet = p >= 0.5
    any_wet = wet.any(axis=0)
    top = ny - 1 - np.argmax(wet[::-1, :], axis=0)  # topmost wet cell per column
    h = np.zeros(nx)
    cols = np.nonzero(any_wet)[0]
    y = top[cols]
    below = p[y, cols]
    above = np.where(y + 1 < ny, p[np.minimum(y + 1, ny - 1), cols], 0.0)
    # crossing between the wet cell y (>= 0.5) and the cell above (< 0.5)
    frac = np.where(below > above, (below - 0.5) / np.maximum(below - above, 1e-300), 0.0)
    h[cols] = y + 0.5 + np.clip(frac, 0.0, 1.0)
    return h


def compare(u, phi, flags, u64, phi64, flags64, nx, ny) -> dict:
    N = nx * ny
    live = np.isin(flags & 7, LIVE) & np.isin(flags64 & 7, LIVE) & ((flags & cases.WALL) == 0)
    m = np.concatenate([live, live])
    du = u.astype(np.float64)[m] - u64[m]
    ref = np.linalg.norm(u64[m])
    l2 = float(np.linalg.norm(du) / ref) if ref > 0 else float("nan")
    ph, ph64 = phi.reshape(ny, nx), phi64.reshape(ny, nx)
    fl, fl64 = flags.reshape(ny, nx), flags64.reshape(ny, nx)
    h, h64 = surface_heights(ph, fl), surface_heights(ph64, fl64)
    solid = (fl & cases.WALL) != 0
    d = np.where(solid, 0.0, ph).sum(axis=0)
    d64 = np.where((fl64 & cases.WALL) != 0, 0.0, ph64).sum(axis=0)
    return {"velocity_l2": l2, "surface_error_cells": float(np.abs(h - h64).mean()),
            "depth_error_cells": float(np.abs(d - d64).mean()), "cells_compared": int(live.sum()),
            "flag_mismatch_cells": int((flags != flags64).sum()), "of_cells": N}


CHECKPOINTS = (500, 1000, 2000, 5000, 10000, 20000, 50000)


def run(scale: int = 4, steps: int = 50_000, u_max: float = 0.25, device: int = -1,
        checkpoints=CHECKPOINTS) -> dict:
    """Runs the three storage precisions side by side and compares FP32 and
    FP16S with FP64 at each checkpoint (and at the end).  Every run also
    reports its own mass drift and its device time."""
    import torch

    c = cases.dam_break(scale)
    out = {"case": c.name, "nx": c.nx, "ny": c.ny, "steps": steps, "tau": c.tau, "g_y": c.fy, "u_max": u_max,
           "modes": "half-way walls, conservative free surface, fused arithmetic, FP64 mass/excess/fill level"}
    names = {64: "fp64", 32: "fp32", 16: "fp16s"}
    solvers, m0, ms = {}, {}, {}
    for prec in (64, 32, 16):
        s = E.Solver(c.flags, free_surface=True, precision=prec, mass_precision=64, tau=c.tau, fy=c.fy,
                     bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, u_max=u_max, device=device)
        solvers[prec], m0[prec], ms[prec] = s, s.total_mass(), 0.0
    series = {"fp32": [], "fp16s": []}
    marks = sorted({k for k in checkpoints if k < steps} | {steps})
    done = 0
    for mark in marks:
        for prec, s in solvers.items():
            st = torch.cuda.ExternalStream(s.stream)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            s.step(mark - done)
            e1.record(st)
            e1.synchronize()
            ms[prec] += e0.elapsed_time(e1)
        done = mark
        ref = solvers[64]
        u64, phi64, fl64 = ref.u.astype(np.float64), ref.phi.astype(np.float64), ref.flags
        for prec in (32, 16):
            s = solvers[prec]
            r = compare(s.u, s.phi.astype(np.float64), s.flags, u64, phi64, fl64, c.nx, c.ny)
            r["step"] = mark
            r["mass_drift"] = (s.total_mass() - m0[prec]) / m0[prec]
            series[names[prec]].append(r)
    for prec, s in solvers.items():
        name = names[prec]
        res = {"mass_drift": (s.total_mass() - m0[prec]) / m0[prec], "finite": s.check_finite(),
               "device_s": round(ms[prec] * 1e-3, 2), "mlups": round(c.cells * steps / (ms[prec] * 1e-3) / 1e6, 1)}
        if prec != 64:
            last = series[name][-1]
            res.update({k: last[k] for k in ("velocity_l2", "surface_error_cells", "depth_error_cells",
                                             "cells_compared", "flag_mismatch_cells", "of_cells")})
            res["series"] = series[name]
        out[name] = res
        s.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--scale", type=int, default=4)
    ap.add_argument("--steps", type=int, default=50_000)
    ap.add_argument("--u-max", type=float, default=0.25)
    a = ap.parse_args(argv)
    print(json.dumps(run(a.scale, a.steps, a.u_max)))


if __name__ == "__main__":
    main()
