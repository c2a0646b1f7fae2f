"""Headless case runner: the counterpart of FlowLB's no-graphics run loops
(``src/cuda/runCuda.cu:460-528``) for the synthetic cases.

    python -m flowlb_b200.run_case --case dam-break --scale 4 --precision 32 --steps 200
    python -m flowlb_b200.run_case --files DIR [--out OUT] [--steps N]

``--files DIR`` is FlowLB's own headless run: DIR/Geometry.txt and
DIR/OptionsCalc.txt set the case up and the VTK results go to
OUT/results_<k>/ (``flb_run_from_files``; ``--steps`` caps the step count).

Prints one JSON line with the device time (CUDA events on the engine's
stream), MLUPS, total mass and the cell census.  ``--profile`` reports the
per-pass device times instead of timing graph-replayed steps.
"""
from __future__ import annotations

import argparse
import json
import time

from . import cases
from . import engine as E

CASES = {
    "channel": lambda a: cases.plain_channel(a.nx or 256, a.ny or 64),
    "probe": lambda a: cases.hbm_probe(a.nx or 8192, a.ny or 2048),
    "dam-break": lambda a: cases.dam_break(a.scale),
    "small-dam-break": lambda a: cases.small_dam_break(a.nx or 96, a.ny or 64),
}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--case", default="dam-break", choices=sorted(CASES))
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--nx", type=int, default=0)
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--precision", type=int, default=32, choices=[16, 32, 64])
    ap.add_argument("--mass-precision", type=int, default=64, choices=[32, 64])
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--bounce-back", default="halfway", choices=["halfway", "implicit"])
    ap.add_argument("--fs-mode", default="conservative", choices=["conservative", "reference"])
    ap.add_argument("--subgrid", action="store_true")
    ap.add_argument("--kernel-variant", type=int, default=0, choices=[0, 1, 2])
    ap.add_argument("--profile", action="store_true", help="per-pass CUDA-event times")
    ap.add_argument("--u-max", type=float, default=0.0, help="velocity limiter (0 = off)")
    ap.add_argument("--arithmetic", default="fused", choices=["fused", "reference"])
    ap.add_argument("--step-mode", default="auto", choices=["auto", "kernels", "persistent"],
                    help="free-surface step form (flb_set_step_mode)")
    ap.add_argument("--files", default="", help="folder with Geometry.txt and OptionsCalc.txt")
    ap.add_argument("--out", default="", help="where --files writes results_<k>/ (default: the folder itself)")
    a = ap.parse_args(argv)
    if a.files:
        import os
        geo, opt = os.path.join(a.files, "Geometry.txt"), os.path.join(a.files, "OptionsCalc.txt")
        import sys
        given = argv if argv is not None else sys.argv[1:]
        capped = any(x == "--steps" or x.startswith("--steps=") for x in given)
        info = E.run_from_files(geo, opt, a.out or a.files, max_steps=a.steps if capped else 0)
        print(json.dumps(info))
        return
    case = CASES[a.case](a)
    s = E.Solver(case.flags, free_surface=case.free_surface, precision=a.precision,
                 mass_precision=a.mass_precision, tau=case.tau, fx=case.fx, fy=case.fy, subgrid=a.subgrid,
                 bounce_back=E.BB_HALFWAY if a.bounce_back == "halfway" else E.BB_IMPLICIT,
                 fs_mode=E.FS_CONSERVATIVE if a.fs_mode == "conservative" else E.FS_REFERENCE,
                 kernel_variant=a.kernel_variant, u_max=a.u_max,
                 arithmetic=E.ARITH_FUSED if a.arithmetic == "fused" else E.ARITH_REFERENCE)
    if case.free_surface:
        s.set_step_mode({"auto": E.STEP_AUTO, "kernels": E.STEP_KERNELS, "persistent": E.STEP_PERSISTENT}[a.step_mode])
    m0 = s.total_mass()
    s.step(a.warmup)
    s.sync()
    out = {"case": case.name, "cells": case.cells, "precision": a.precision, "steps": a.steps,
           "step_form": "persistent kernel" if case.free_surface and s.persistent else "per-pass kernels"}
    if a.profile:
        passes = s.profile_steps(a.steps)
        total = sum(passes.values())
        out["pass_ms_per_step"] = {k: round(v / a.steps, 5) for k, v in passes.items()}
        out["mlups"] = round(case.cells * a.steps / (total * 1e-3) / 1e6, 1)
    else:
        import torch
        st = torch.cuda.ExternalStream(s.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        ev0.record(st)
        s.step(a.steps)
        ev1.record(st)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        out["device_ms"] = round(ms, 3)
        out["wall_s"] = round(time.perf_counter() - t0, 3)
        out["mlups"] = round(case.cells * a.steps / (ms * 1e-3) / 1e6, 1)
    out["mass_rel_drift"] = (s.total_mass() - m0) / m0 if m0 else None
    out["cells_by_type"] = s.cell_counts()
    out["finite"] = s.check_finite()
    out["launches"] = s.launches
    print(json.dumps(out))
    s.close()


if __name__ == "__main__":
    main()
