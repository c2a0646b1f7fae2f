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


def _engine_ms(solver, n):
    import torch

    st = torch.cuda.ExternalStream(solver.stream)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    solver.step(n)
    b.record(st)
    b.synchronize()
    return a.elapsed_time(b)


def _record(line):
    """Prints a timing line; appends it as JSON to $FLB_TIMING_OUT when set."""
    import json
    import os

    print(json.dumps(line))
    path = os.environ.get("FLB_TIMING_OUT")
    if path:
        with open(path, "a") as fp:
            fp.write(json.dumps(line) + "\n")


TIMING_BUILD = "timing" if O.ref_cuda_timing_available() else "parity"


def test_engine_outpaces_reference_kernels_single_phase_8192x2048():
    """The engine in the reference's own modes (implicit walls, reference
    arithmetic) against FlowLB's CUDA kernels on the same GPU, 8192x2048 plain
    channel, FP32: equal populations after the same 220 steps (against the
    kernels as written, no contraction), and a faster step (device time of the
    last 200 steps of each; the reference timed in its own build, debug
    printf calls compiled out)."""
    import flowlb_b200.engine as E

    c = cases.hbm_probe(8192, 2048)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32_M32, tau=c.tau, fx=c.fx))
    st0 = snapshot(o, False)
    o.close()
    nofma_ms, ref = O.ref_cuda_time(st0, c.nx, c.ny, 32, False, c.tau, c.fx, 0.0, warm=20, nsteps=200)
    ref_ms, _ = O.ref_cuda_time(st0, c.nx, c.ny, 32, False, c.tau, c.fx, 0.0, warm=20, nsteps=200,
                                build=TIMING_BUILD)
    s = E.Solver(c.flags, precision=32, mass_precision=32, tau=c.tau, fx=c.fx, bounce_back=E.BB_IMPLICIT,
                 arithmetic=E.ARITH_REFERENCE, device=0)
    s.step(20)
    s.sync()
    eng_ms = _engine_ms(s, 200)
    assert exact_equal(s.f, ref["f"]), first_mismatch(s.f, ref["f"])
    s.close()
    # the engine's own defaults (half-way walls, fused arithmetic)
    d = E.Solver(c.flags, precision=32, tau=c.tau, fx=c.fx, device=0)
    d.step(20)
    d.sync()
    def_ms = _engine_ms(d, 200)
    d.close()
    mlups = lambda ms: c.cells * 200 / (ms * 1e-3) / 1e6  # noqa: E731
    _record({"case": "single phase 8192x2048 FP32, 200 steps", "reference_build": TIMING_BUILD,
             "reference_kernels_mlups": round(mlups(ref_ms), 1),
             "reference_kernels_no_contraction_mlups": round(mlups(nofma_ms), 1),
             "engine_reference_modes_mlups": round(mlups(eng_ms), 1), "engine_defaults_mlups": round(mlups(def_ms), 1),
             "speedup_reference_modes": round(ref_ms / eng_ms, 2), "speedup_defaults": round(ref_ms / def_ms, 2)})
    assert eng_ms < ref_ms


def test_engine_outpaces_reference_kernels_dam_break_2048x512():
    """The free-surface step in the reference's modes against FlowLB's five
    CUDA kernels per step on the same GPU, 2048x512 dam break, FP32 (mass in
    FP32 as in the reference): device time of 200 steps after 20 (the
    reference in its own build, debug printf calls compiled out)."""
    import flowlb_b200.engine as E

    c = cases.dam_break(1)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32_M32, free_surface=True, tau=c.tau, fy=c.fy))
    st0 = snapshot(o, True)
    o.close()
    nofma_ms, _ = O.ref_cuda_time(st0, c.nx, c.ny, 32, True, c.tau, 0.0, c.fy, warm=20, nsteps=200)
    ref_ms, _ = O.ref_cuda_time(st0, c.nx, c.ny, 32, True, c.tau, 0.0, c.fy, warm=20, nsteps=200,
                                build=TIMING_BUILD)
    s = E.Solver(c.flags, free_surface=True, precision=32, mass_precision=32, tau=c.tau, fy=c.fy,
                 bounce_back=E.BB_IMPLICIT, fs_mode=E.FS_REFERENCE, arithmetic=E.ARITH_REFERENCE, device=0)
    s.step(20)
    s.sync()
    eng_ms = _engine_ms(s, 200)
    s.close()
    d = E.Solver(c.flags, free_surface=True, precision=32, mass_precision=64, tau=c.tau, fy=c.fy, u_max=0.25,
                 device=0)
    d.step(20)
    d.sync()
    def_ms = _engine_ms(d, 200)
    d.close()
    mlups = lambda ms: c.cells * 200 / (ms * 1e-3) / 1e6  # noqa: E731
    _record({"case": "free-surface dam break 2048x512 FP32, 200 steps", "reference_build": TIMING_BUILD,
             "reference_kernels_mlups": round(mlups(ref_ms), 1),
             "reference_kernels_no_contraction_mlups": round(mlups(nofma_ms), 1),
             "engine_reference_modes_mlups": round(mlups(eng_ms), 1),
             "engine_defaults_fp64_mass_mlups": round(mlups(def_ms), 1),
             "speedup_reference_modes": round(ref_ms / eng_ms, 2), "speedup_defaults": round(ref_ms / def_ms, 2)})
    assert eng_ms < ref_ms


@pytest.mark.parametrize("prec", [32, 64])
def test_isoline_matches_reference_kernel(prec):
    """flb_viz_isoline against the reference's own d_CreateIsoSurfaceVector2D
    (src/cuda/cudaIsosurface.cuh:33-199, cudaIsosurface.cu:16-76, compiled in
    place) on the velocity magnitude of a free-surface state: whole domain,
    camera windows and up- and down-scaled images.  The camera bounds stay
    inside the lattice, where every pixel the reference writes lies inside
    the image (its surface traps out of range).  The engine takes the
    magnitude as sqrt(x*x + y*y) rounded per operation, the reference calls
    hypotf: the two may differ in the last bit of a node value, which can move
    a line end across a pixel boundary, so a few pixels may differ; the test
    counts them and holds them to 0.5 % of the reference's line pixels."""
    from flowlb_b200 import engine as E

    c = cases.small_dam_break(160, 96)
    s = E.Solver(c.flags, free_surface=True, precision=prec, mass_precision=64, tau=0.55, fy=-5e-4, u_max=0.25)
    s.step(400)
    u = s.u
    speed = np.hypot(u[:s.N].astype(np.float64), u[s.N:].astype(np.float64))
    assert np.isfinite(speed).all()
    total_diff = total_line = 0
    for frac in (0.25, 0.5):
        iso = float(np.quantile(speed[speed > 0], frac))
        for (w, h), b in (((160, 96), (0, 160, 0, 96)), ((480, 288), (0, 160, 0, 96)), ((64, 40), (0, 160, 0, 96)),
                          ((300, 200), (20, 130, 10, 80)), ((97, 61), (40, 160, 0, 50))):
            got = s.viz_isoline(E.FIELD_U, iso, w, h, b)
            ref = O.ref_cuda_isoline(u, s.nx, s.ny, prec, iso, w, h, b)
            line = int((ref != 0).sum())
            diff = int((got != ref).sum())
            assert line > 0
            total_line += line
            total_diff += diff
            assert diff <= max(4, 0.005 * line), (iso, w, h, b, diff, line)
    print(f"iso-line pixels differing from the reference kernel: {total_diff} of {total_line}")
    s.close()
