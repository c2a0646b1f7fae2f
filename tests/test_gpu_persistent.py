"""The persistent free-surface step (one cooperative kernel per graph of
steps, passes separated by grid barriers) against the per-pass kernels and
the oracle, and its failure detection.

Both forms run the same per-cell code, so every field must be equal bit for
bit whichever form ran which steps.
"""
import numpy as np
import pytest

from conftest import exact_equal, first_mismatch
from flowlb_b200 import cases
from flowlb_b200 import engine as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = (("f", E.FIELD_F), ("rho", E.FIELD_RHO), ("u", E.FIELD_U), ("flags", E.FIELD_FLAGS),
          ("mass", E.FIELD_MASS), ("excess", E.FIELD_EXCESS), ("phi", E.FIELD_PHI))


def _same(a, b, what):
    for name, fid in FIELDS:
        x, y = a.read(fid), b.read(fid)
        assert exact_equal(x, y), f"{what} {name}: {first_mismatch(x, y)}"


VARIANTS = [(32, 64, E.BB_HALFWAY, E.FS_CONSERVATIVE, E.ARITH_FUSED),
            (64, 64, E.BB_HALFWAY, E.FS_CONSERVATIVE, E.ARITH_FUSED),
            (16, 64, E.BB_HALFWAY, E.FS_CONSERVATIVE, E.ARITH_FUSED),
            (32, 32, E.BB_IMPLICIT, E.FS_REFERENCE, E.ARITH_REFERENCE),
            (64, 64, E.BB_IMPLICIT, E.FS_REFERENCE, E.ARITH_REFERENCE),
            (32, 64, E.BB_IMPLICIT, E.FS_CONSERVATIVE, E.ARITH_REFERENCE)]


@pytest.mark.parametrize("prec,mprec,bb,fsm,arith", VARIANTS, ids=lambda v: str(v))
def test_persistent_equals_per_pass_kernels(prec, mprec, bb, fsm, arith):
    """Small dam break under strong gravity (the surge reaches the far wall):
    persistent and per-pass forms stay equal over 700 steps, with runs of 32
    and 2 steps and single steps interleaved."""
    c = cases.small_dam_break(160, 72)
    kw = dict(free_surface=True, precision=prec, mass_precision=mprec, tau=0.55, fy=-5e-4, bounce_back=bb,
              fs_mode=fsm, arithmetic=arith, u_max=0.25)
    a = E.Solver(c.flags, **kw)
    b = E.Solver(c.flags, **kw)
    a.set_step_mode(E.STEP_PERSISTENT)
    b.set_step_mode(E.STEP_KERNELS)
    assert a.persistent and not b.persistent
    for n in (1, 67, 3, 200, 5, 424):
        a.step(n)
        b.step(n)
        _same(a, b, f"t={a.t}")
    a.close()
    b.close()


def test_persistent_dam_break_2048x512_equals_oracle():
    """The bench workload for 600 steps in the persistent form against the
    FP32 oracle twin."""
    c = cases.dam_break(1)
    kw = dict(tau=c.tau, fy=c.fy, u_max=0.25)
    s = E.Solver(c.flags, free_surface=True, precision=32, mass_precision=64, **kw)
    s.set_step_mode(E.STEP_PERSISTENT)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32, free_surface=True, bb=O.BB_HALFWAY, fs_mode=O.FS_CONSERVATIVE,
                                         arithmetic=O.ARITH_FUSED, **kw))
    for n in (300, 300):
        s.step(n)
        o.step(n)
        for name, a, b in (("f", s.f, o.f64().astype(np.float32)), ("flags", s.flags, o.flags),
                           ("mass", s.mass, o.mass), ("phi", s.phi, o.phi), ("excess", s.excess, o.excess),
                           ("rho", s.rho, o.rho), ("u", s.u, o.u)):
            assert exact_equal(a, b), f"t={o.t} {name}: {first_mismatch(a, b)}"
    s.close()
    o.close()


def test_persistent_on_many_super_tiles_equals_per_pass():
    """More than 4096 super-tiles (the per-pass flag kernel switches to
    32-wide tiles there) with the persistent form forced: same results."""
    c = cases.small_dam_break(4352, 1024)  # 34 x 128 = 4352 super-tiles
    flags = c.flags
    kw = dict(free_surface=True, precision=32, mass_precision=64, tau=c.tau, fy=c.fy, u_max=0.25)
    a = E.Solver(flags, **kw)
    b = E.Solver(flags, **kw)
    a.set_step_mode(E.STEP_PERSISTENT)
    b.set_step_mode(E.STEP_KERNELS)
    for n in (1, 99):
        a.step(n)
        b.step(n)
    _same(a, b, "t=100")
    a.close()
    b.close()


def test_step_mode_is_validated():
    ch = cases.plain_channel(64, 16)
    s = E.Solver(ch.flags, precision=32, tau=ch.tau, fx=ch.fx)
    with pytest.raises(E.FlowLBError) as ei:
        s.set_step_mode(E.STEP_PERSISTENT)  # single phase has no persistent form
    assert ei.value.status == 4
    s.set_step_mode(E.STEP_AUTO)
    with pytest.raises(E.FlowLBError) as ei:
        s.set_step_mode(7)
    assert ei.value.status == 1
    s.close()


def test_persistent_barrier_wait_runs_out_and_reset_recovers(monkeypatch):
    """Failure detection of the grid barriers, made on the host: with
    FLB_PERSIST_SKIP_ARRIVAL=1 one CTA never arrives, so every wait runs out
    after a short limit (4,096 polls) and the kernel leaves.  flb_sync reports
    FLB_ERR_CUDA, stepping is refused until flb_reset, and after the reset the
    handle steps bit-equal to a fresh one.  The reference has no failure
    handling here: its CUDA error check exits the process
    (src/cuda/cudaUtils.cuh:17-26)."""
    c = cases.small_dam_break(96, 64)
    kw = dict(free_surface=True, precision=32, mass_precision=64, tau=c.tau, fy=c.fy)
    s = E.Solver(c.flags, **kw)
    s.set_step_mode(E.STEP_PERSISTENT)
    s.step(1)  # the first step after set-up runs per pass
    s.set_wait_limit(4096)
    monkeypatch.setenv("FLB_PERSIST_SKIP_ARRIVAL", "1")
    s.step(40)  # from an odd t: one single step, then a graph of 32 and ...
    with pytest.raises(E.FlowLBError) as ei:
        s.sync()
    assert ei.value.status == 2  # FLB_ERR_CUDA
    with pytest.raises(E.FlowLBError) as ei:
        s.step(1)
    assert ei.value.status == 2
    monkeypatch.delenv("FLB_PERSIST_SKIP_ARRIVAL")
    s.reset(c.flags)
    s.set_wait_limit(0)
    ref = E.Solver(c.flags, **kw)
    ref.set_step_mode(E.STEP_KERNELS)
    s.step(77)
    ref.step(77)
    s.sync()
    _same(s, ref, "after reset")
    s.close()
    ref.close()
