"""Failure detection through the C ABI, with every failure made on the host.

Nothing here faults, traps or hangs a GPU: non-finite populations are written
into a case through flb_write_field, and an allocation failure is injected by
the engine's host-side hook (FLB_FAIL_ALLOC_AT=k fails the k-th device
allocation of a creation without attempting it).  The library must report
each through its status codes, free what it allocated, and stay usable."""
import gc
import os

import numpy as np
import pytest

from conftest import exact_equal
from flowlb_b200 import cases
from flowlb_b200 import engine as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [32, 64, 16])
@pytest.mark.parametrize("value", [np.nan, np.inf], ids=["nan", "inf"])
def test_non_finite_population_is_reported(require_gpu, prec, value):
    c = cases.plain_channel(64, 32)
    s = E.Solver(c.flags, precision=prec, tau=c.tau, fx=c.fx, device=0)
    s.step(3)
    assert s.check_finite()
    good = s.f
    bad = good.copy()
    fluid = np.flatnonzero(c.flags.ravel() == cases.FLUID)
    cell = int(fluid[len(fluid) // 2])
    bad[cell + 5 * s.N] = value
    s.write(E.FIELD_F, bad)
    assert not s.check_finite()
    with pytest.raises(E.FlowLBError) as ei:
        s._check(E.load_library().flb_check_finite(s.handle))
    assert ei.value.status == 6 and ": 1 cells hold" in str(ei.value)  # FLB_ERR_NONFINITE
    # a population of a wall cell is not part of the state: not reported
    wall = int(np.flatnonzero(c.flags.ravel() == cases.WALL)[0])
    s.write(E.FIELD_F, good)
    assert s.check_finite()
    bad = good.copy()
    bad[wall] = value
    s.write(E.FIELD_F, bad)
    assert s.check_finite()
    # the handle stays usable: the original state steps on as before (FP16
    # storage is read back decoded, and re-encoding a decoded value is not
    # exact for the smallest deviations, so there only finiteness is checked)
    s.write(E.FIELD_F, good)
    s.step(4)
    assert s.check_finite()
    if prec != 16:
        ref = E.Solver(c.flags, precision=prec, tau=c.tau, fx=c.fx, device=0)
        ref.step(7)
        assert exact_equal(s.f, ref.f)
        ref.close()
    s.close()


def _free_bytes(torch):
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info(0)[0]


@pytest.mark.parametrize("fs", [False, True], ids=["single-phase", "free-surface"])
def test_injected_allocation_failure_frees_everything(require_gpu, fs, monkeypatch):
    """Every allocation of a creation in turn fails: flb_create returns
    FLB_ERR_OUT_OF_MEMORY, gives nothing back, and leaves the device's free
    memory where it was; without the hook the same creation succeeds."""
    import torch

    c = cases.small_dam_break(512, 256) if fs else cases.plain_channel(512, 256)
    kw = dict(free_surface=fs, precision=32, tau=c.tau, fx=c.fx, fy=c.fy, device=0)
    # the context and every kernel this case launches (loaded lazily on first
    # use) are loaded once, outside the measurement
    w = E.Solver(c.flags, **kw)
    w.step(8)
    w.close()
    # handles left by earlier tests in reference cycles are freed now, not
    # by a collection in the middle of the measurement
    gc.collect()
    gc.disable()
    try:
        _allocation_failures(torch, c, kw, monkeypatch)
    finally:
        gc.enable()


def _allocation_failures(torch, c, kw, monkeypatch):
    before = _free_bytes(torch)
    failures = 0
    for k in range(1, 40):
        monkeypatch.setenv("FLB_FAIL_ALLOC_AT", str(k))
        try:
            s = E.Solver(c.flags, **kw)
        except E.FlowLBError as e:
            assert e.status == 3, str(e)  # FLB_ERR_OUT_OF_MEMORY
            failures += 1
            # 2 MiB: the granularity at which the driver reports free memory
            assert abs(_free_bytes(torch) - before) <= 2 << 20
            continue
        s.close()
        break  # k is past the last allocation: creation succeeded
    else:
        pytest.fail("every injected position failed; the hook never ran out of allocations")
    assert failures >= 10  # populations, fields, flags, lists, scratch ...
    monkeypatch.delenv("FLB_FAIL_ALLOC_AT")
    s = E.Solver(c.flags, **kw)
    s.step(8)
    assert s.check_finite()
    s.close()
    assert abs(_free_bytes(torch) - before) <= 2 << 20
    assert "FLB_FAIL_ALLOC_AT" not in os.environ


@pytest.mark.parametrize("where,msg", [("last", "inlet in the last cell"), ("first", "outlet in the first cell")])
def test_inlet_outlet_placement_is_checked(require_gpu, where, msg):
    """An inlet takes its density from the next cell and an outlet its velocity
    from the previous one, so an inlet in the last cell or an outlet in the
    first is refused with FLB_ERR_INVALID_ARGUMENT, at creation and at a
    reset; a valid reset of the same handle works afterwards."""
    c = cases.plain_channel(64, 16)
    bad = c.flags.copy()
    if where == "last":
        bad.flat[-1] = cases.INLET | cases.FLUID
    else:
        bad.flat[0] = cases.OUTLET | cases.FLUID
    with pytest.raises(E.FlowLBError) as ei:
        E.Solver(bad, free_surface=False, precision=32, tau=c.tau, fx=c.fx, device=0)
    assert ei.value.status == 1  # FLB_ERR_INVALID_ARGUMENT (the reason goes to stderr: no handle exists)
    s = E.Solver(c.flags, free_surface=False, precision=32, tau=c.tau, fx=c.fx, device=0)
    with pytest.raises(E.FlowLBError) as ei:
        s.reset(bad)
    assert ei.value.status == 1 and msg in str(ei.value)
    s.reset(c.flags)
    s.step(4)
    assert s.check_finite()
    s.close()
