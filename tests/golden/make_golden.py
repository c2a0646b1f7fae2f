"""Generates the golden fixtures of tests/golden/ from the reference's own code.

Two sources, both compiled from the FlowLB sources in place by oracle/Makefile:

* ``--host``: FlowLB's host initialisation (initFields, initFreeSurfaceFlags,
  initFreeSurfaceFields; oracle/_ref/libflbref_host.so).  Runs on any machine
  that has the reference tree.
* ``--cuda``: FlowLB's CUDA kernels built with --fmad=false
  (oracle/_ref/libflbref_cuda.so).  Needs a GPU; the library is prebuilt, the
  reference tree is not read.
    - single phase: the reference loop stepped N times from the initial state;
    - free surface: the reference kernels race (FS_1's reconstruction store vs
      a neighbour's outgoing load; FS_4's neighbour count vs a neighbour's flag
      conversion), so a multi-step reference trajectory is not reproducible.
      Instead, along the oracle's own (deterministic) trajectory, each of the
      five reference kernels is applied once to the oracle's state at a few
      sampled steps and the fields that kernel writes are recorded.

Usage:  python tests/golden/make_golden.py --host
        python tests/golden/make_golden.py --cuda [--out DIR]
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

FS_SAMPLE_STEPS = (0, 9, 23)
# fields each reference kernel writes (f of FS_1/FS_3 stored sparsely)
KERNEL_FIELDS = {
    O.K_FS1: ("mass", "f~"),
    O.K_STREAM_COLLIDE: ("f", "rho", "u", "flags"),
    O.K_FS2: ("flags",),
    O.K_FS3: ("flags", "f~"),
    O.K_FS4: ("flags", "mass", "excess", "phi"),
}
KNAME = {O.K_FS1: "fs1", O.K_STREAM_COLLIDE: "sc", O.K_FS2: "fs2", O.K_FS3: "fs3", O.K_FS4: "fs4"}


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


def snapshot(o, fs=True):
    st = dict(f=o.f.copy(), rho=o.rho.copy(), u=o.u.copy(), flags=o.flags.copy())
    if fs:
        st.update(mass=o.mass.copy(), excess=o.excess.copy(), phi=o.phi.copy())
    return st


def free_surface_oracle(flags, prec, tau, fx, fy):
    var = O.F32_M32 if prec == 32 else O.F64
    return O.Oracle(flags, O.OracleConfig(variant=var, free_surface=True, tau=tau, fx=fx, fy=fy))


def make_cuda(out_dir=HERE):
    os.makedirs(out_dir, exist_ok=True)
    for name, flags, fs, tau, fx, fy, steps in golden_cases():
        for prec in (32, 64):
            init = dict(np.load(os.path.join(HERE, f"init_{name}_p{prec}.npz")))
            geo = init.pop("geometry")
            ny, nx = geo.shape
            if not fs:
                out = O.ref_cuda_run(init, nx, ny, prec, fs, tau, fx, fy, t0=0, nsteps=steps)
                path = os.path.join(out_dir, f"step_{name}_p{prec}_t{steps}.npz")
                np.savez_compressed(path, geometry=geo, tau=tau, fx=fx, fy=fy, steps=steps, **out)
                print("wrote", path)
                continue
            o = free_surface_oracle(geo, prec, tau, fx, fy)
            rec = dict(geometry=geo, tau=tau, fx=fx, fy=fy, sample_steps=np.array(FS_SAMPLE_STEPS))
            for step in range(max(FS_SAMPLE_STEPS) + 1):
                for kid in (O.K_FS1, O.K_STREAM_COLLIDE, O.K_FS2, O.K_FS3, O.K_FS4):
                    if step in FS_SAMPLE_STEPS:
                        st = snapshot(o)
                        ref = O.ref_cuda_run(st, nx, ny, prec, True, tau, fx, fy, t0=o.t, kernel_id=kid)
                        for fld in KERNEL_FIELDS[kid]:
                            key = f"s{step}_{KNAME[kid]}_"
                            if fld == "f~":
                                changed = np.nonzero(ref["f"] != st["f"])[0]
                                rec[key + "f_idx"] = changed.astype(np.int32)
                                rec[key + "f_val"] = ref["f"][changed]
                            else:
                                rec[key + fld] = ref[fld]
                    o.kernel(kid)
                o.t = o.t + 1
            path = os.path.join(out_dir, f"kernels_{name}_p{prec}.npz")
            np.savez_compressed(path, **rec)
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
