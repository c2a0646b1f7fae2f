"""Generates the golden fixtures of tests/golden/ from the reference's own code.

Two sources, both compiled from the FlowLB sources in place by oracle/Makefile:

* ``--host``: FlowLB's host initialisation (initFields, initFreeSurfaceFlags,
  initFreeSurfaceFields; oracle/_ref/libflbref_host.so).  Runs on any machine
  that has the reference tree.
* ``--cuda``: FlowLB's CUDA kernels built with --fmad=false
  (oracle/_ref/libflbref_cuda.so) stepping small cases from that initial
  state.  Needs a GPU; the library is prebuilt, the reference tree is not read.

Usage:  python tests/golden/make_golden.py --host
        python tests/golden/make_golden.py --cuda
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from flowlb_b200 import cases  # noqa: E402
from oracle import oracle as O  # noqa: E402

# Small cases: (name, geometry flags, free surface, tau, fx, fy, steps)
def golden_cases():
    ch = cases.plain_channel(48, 24)
    db = cases.small_dam_break(40, 32)
    return [
        ("channel_48x24", ch.flags, False, ch.tau, 1e-4, 0.0, 64),
        ("dambreak_40x32", db.flags, True, db.tau, 0.0, -5e-4, 24),
    ]


def make_host():
    for name, flags, fs, *_ in golden_cases():
        for prec in (32, 64):
            st = O.ref_host_init(flags, prec, fs)
            path = os.path.join(HERE, f"init_{name}_p{prec}.npz")
            np.savez_compressed(path, geometry=flags, **st)
            print("wrote", path)


def make_cuda(out_dir=HERE):
    os.makedirs(out_dir, exist_ok=True)
    for name, flags, fs, tau, fx, fy, steps in golden_cases():
        for prec in (32, 64):
            init = dict(np.load(os.path.join(HERE, f"init_{name}_p{prec}.npz")))
            geo = init.pop("geometry")
            ny, nx = geo.shape
            out = O.ref_cuda_run(init, nx, ny, prec, fs, tau, fx, fy, t0=0, nsteps=steps)
            path = os.path.join(out_dir, f"step_{name}_p{prec}_t{steps}.npz")
            np.savez_compressed(path, geometry=geo, tau=tau, fx=fx, fy=fy, steps=steps, **out)
            print("wrote", path)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--host", action="store_true")
    ap.add_argument("--cuda", action="store_true")
    ap.add_argument("--out", default=HERE, help="output directory of --cuda")
    a = ap.parse_args()
    if a.host:
        make_host()
    if a.cuda:
        make_cuda(a.out)
