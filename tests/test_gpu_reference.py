"""GPU pin of the oracle against FlowLB's own CUDA kernels.

oracle/_ref/libflbref_cuda.so is the reference's src/cuda/lbmKernel2D.cu and
cudaInitData.cu compiled unmodified (--fmad=false) with a launch harness.  The
oracle in reference mode must reproduce each reference kernel exactly.  Where
the reference kernels race (FS_4's neighbour count reads flags that
neighbours rewrite in the same launch) the reference result must equal the
oracle's result with either the converted ("post") or unconverted ("pre")
neighbour flags.
"""
import numpy as np
import pytest

from conftest import exact_equal, first_mismatch
from flowlb_b200 import cases
from oracle import oracle as O

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not O.ref_cuda_available(), reason="reference CUDA lib missing")]

VAR = {32: O.F32_M32, 64: O.F64}


def snapshot(o, fs):
    st = dict(f=o.f.copy(), rho=o.rho.copy(), u=o.u.copy(), flags=o.flags.copy())
    if fs:
        st.update(mass=o.mass.copy(), excess=o.excess.copy(), phi=o.phi.copy())
    return st


def compare(ref, o, fs, what):
    keys = ["f", "rho", "u", "flags"] + (["mass", "excess", "phi"] if fs else [])
    for k in keys:
        assert exact_equal(ref[k], getattr(o, k)), f"{what} {k}: {first_mismatch(ref[k], getattr(o, k))}"


@pytest.mark.parametrize("prec", [32, 64])
def test_single_phase_trajectory_matches_reference(prec):
    c = cases.plain_channel(96, 40)
    o = O.Oracle(c.flags, O.OracleConfig(variant=VAR[prec], tau=c.tau, fx=1e-4))
    ref = O.ref_cuda_run(snapshot(o, False), c.nx, c.ny, prec, False, c.tau, 1e-4, 0.0, t0=0, nsteps=301)
    o.step(301)
    compare(ref, o, False, f"p{prec} t=301")


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("opts", [dict(subgrid=True), dict(collision=1, use_force=False)], ids=["smagorinsky", "trt"])
def test_single_phase_options_match_reference(prec, opts):
    c = cases.plain_channel(64, 24)
    o = O.Oracle(c.flags, O.OracleConfig(variant=VAR[prec], tau=0.53, fx=2e-4, **opts))
    ref = O.ref_cuda_run(snapshot(o, False), c.nx, c.ny, prec, False, 0.53, 2e-4, 0.0, t0=0, nsteps=57,
                         collision=opts.get("collision", 0), subgrid=opts.get("subgrid", False),
                         use_force=opts.get("use_force", True))
    o.step(57)
    compare(ref, o, False, f"p{prec} {opts}")


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("mode", ["implicit", "tall"])
def test_free_surface_kernels_match_reference_along_a_trajectory(prec, mode):
    """At every step of a dam-break trajectory, each of the five reference
    kernels applied to the oracle's state gives the oracle's output; for the
    two racing kernels each cell matches one of the two interleavings."""
    from refcheck import check_kernel, snapshot
    c = cases.small_dam_break(64, 48) if mode == "implicit" else cases.small_dam_break(48, 96)
    cfg = O.OracleConfig(variant=VAR[prec], free_surface=True, tau=c.tau, fy=c.fy * (4 if mode == "tall" else 1))
    o = O.Oracle(c.flags, cfg)
    raced = 0
    for step in range(60):
        for kid in (O.K_FS1, O.K_STREAM_COLLIDE, O.K_FS2, O.K_FS3, O.K_FS4):
            st = snapshot(o)
            ref = O.ref_cuda_run(st, c.nx, c.ny, prec, True, cfg.tau, 0.0, cfg.fy, t0=o.t, kernel_id=kid)
            res = check_kernel(c.flags, cfg, st, o.t, kid, ref, f"p{prec} step {step} kernel {kid}")
            raced += res["raced"]
            o.kernel(kid)
        o.t = o.t + 1
    print("cells decided by a race in the reference:", raced)
