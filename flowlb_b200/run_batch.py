"""Runs the batched culvert ensemble (``flb_batch_*``) from the command line.

    python -m flowlb_b200.run_batch --cases 512 --steps 5000
    python -m flowlb_b200.run_batch --cases 128 --steps 20 --shape team,45,3,512

The ensemble is ``cases.ensemble()`` (seeded single-phase culvert channels);
``--cases`` takes the first n of the 512.  Without ``--shape`` the launch shape
is chosen by the batch's own timed search (``--autotune`` probe steps); with it
the search is skipped and the shape "mode,CTAs per group,groups,threads[,vector]"
is set (``flb_batch_set_launch``; "streams,1,S,0" for the streams form on S
streams).  Prints one JSON line: the shape that ran,
the wall time of the stepped launch (after a 2-step warm-up) and its rate.
"""
from __future__ import annotations

import argparse
import json
import time

from . import cases
from . import engine as E


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--cases", type=int, default=512)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--autotune", type=int, default=1, help="probe steps of the shape search (1: 100)")
    ap.add_argument("--shape", default="", help="mode,group,groups,threads[,vector]")
    a = ap.parse_args(argv)
    ens = cases.ensemble()[:a.cases]
    b = E.Batch([(e.flags, e.tau, e.fx, 0.0) for e in ens], autotune=0 if a.shape else a.autotune)
    if a.shape:
        parts = a.shape.split(",")
        b.set_launch(parts[0], int(parts[1]), int(parts[2]), int(parts[3]),
                     vector=len(parts) > 4 and parts[4] in ("1", "vector", "true"))
    b.step(2)
    b.sync()
    t0 = time.perf_counter()
    b.step(a.steps)
    b.sync()
    dt = time.perf_counter() - t0
    info = b.info()
    print(json.dumps({"cases": len(ens), "steps": a.steps, "wall_s": round(dt, 4),
                      "cases_per_s": round(len(ens) / dt * a.steps / 5000.0, 2) if a.steps else None,
                      "glups": round(info["cells"] * a.steps / dt / 1e9, 2), "shape": info}))
    b.close()


if __name__ == "__main__":
    main()
