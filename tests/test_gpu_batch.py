"""Batched ensemble (flb_batch_*) against one handle per case.

The batch kernel updates cells with the same per-cell code as the
single-case kernels, so after the same number of steps every case must equal
its own Solver run bit for bit (populations, density, velocity, flags).
"""
import numpy as np
import pytest

from conftest import exact_equal, first_mismatch
from flowlb_b200 import cases
from flowlb_b200 import engine as E

pytestmark = pytest.mark.gpu


def _small_ensemble(n, seed):
    """Seeded cases of the ensemble's kind, scaled down (and some tiny ones)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nx = int(rng.integers(9, 300))
        ny = int(rng.integers(5, 70))
        w = max(1, int(round(rng.uniform(0.05, 0.2) * nx)))
        h = max(1, int(round(rng.uniform(0.2, 0.6) * ny)))
        x0 = nx // 2 - w // 2
        flags = cases.channel_with_block(nx, ny, x0, x0 + w, min(ny - 2, 1 + h))
        tau = float(np.float32(rng.uniform(0.52, 0.8)))
        gx = float(np.float32(10.0 ** rng.uniform(-7.0, -4.0)))
        out.append((flags, tau, gx, 0.0))
    return out


@pytest.mark.parametrize("bb", [E.BB_HALFWAY, E.BB_IMPLICIT], ids=["halfway", "implicit"])
@pytest.mark.parametrize("arith", [E.ARITH_FUSED, E.ARITH_REFERENCE], ids=["fused", "ref-arith"])
@pytest.mark.parametrize("autotune", [0, 4], ids=["fixed", "tuned"])
def test_batch_matches_single_handles(bb, arith, autotune):
    ens = _small_ensemble(23, 20261203)
    b = E.Batch(ens, bounce_back=bb, arithmetic=arith, autotune=autotune)
    info = b.info()
    assert info["cases"] == len(ens) and info["tuned"] == bool(autotune)
    for n in (1, 37, 64):  # odd and even starting parities, one launch each
        b.step(n)
    b.sync()
    assert b.info()["t"] == 102
    for i, (flags, tau, gx, gy) in enumerate(ens):
        s = E.Solver(flags, precision=32, tau=tau, fx=gx, fy=gy, bounce_back=bb, arithmetic=arith)
        s.step(102)
        for name, fid, ref in (("f", E.FIELD_F, s.f), ("rho", E.FIELD_RHO, s.rho), ("u", E.FIELD_U, s.u),
                               ("flags", E.FIELD_FLAGS, s.flags)):
            got = b.read(i, fid)
            assert exact_equal(got, ref), f"case {i} {flags.shape} {name}: {first_mismatch(got, ref)}"
        s.close()
    b.reset()
    assert b.info()["t"] == 0
    b.close()


@pytest.mark.parametrize("bb", [E.BB_HALFWAY, E.BB_IMPLICIT], ids=["halfway", "implicit"])
@pytest.mark.parametrize("arith", [E.ARITH_FUSED, E.ARITH_REFERENCE], ids=["fused", "ref-arith"])
@pytest.mark.parametrize("shape", [("team", 3, 7, 512), ("team", 1, 23, 256), ("cluster", 8, 2, 512)],
                         ids=lambda v: f"{v[0]}{v[1]}x{v[2]}t{v[3]}")
def test_batch_vector_path_matches_single_handles(bb, arith, shape):
    """The vector data path (four cells per thread, rows padded to a multiple
    of four cells) on widths of every residue mod 4, narrower than a group,
    and wider than one 128-cell warp segment: every case equals its own
    handle bit for bit, from both step parities."""
    ens = _small_ensemble(23, 4321)
    ens[0] = (cases.channel_with_block(3, 7, 1, 2, 2), 0.6, 1e-5, 0.0)
    ens[1] = (cases.channel_with_block(131, 9, 60, 70, 4), 0.55, 2e-5, 0.0)
    ens[2] = (cases.channel_with_block(258, 11, 100, 130, 6), 0.7, 1e-5, 0.0)
    b = E.Batch(ens, bounce_back=bb, arithmetic=arith, autotune=0)
    b.set_launch(*shape, vector=True)
    assert b.info()["vector"]
    for n in (1, 36, 29):
        b.step(n)
    b.sync()
    for i, (flags, tau, gx, gy) in enumerate(ens):
        s = E.Solver(flags, precision=32, tau=tau, fx=gx, fy=gy, bounce_back=bb, arithmetic=arith)
        s.step(66)
        for name, fid, ref in (("f", E.FIELD_F, s.f), ("rho", E.FIELD_RHO, s.rho), ("u", E.FIELD_U, s.u),
                               ("flags", E.FIELD_FLAGS, s.flags)):
            got = b.read(i, fid)
            assert exact_equal(got, ref), f"case {i} {flags.shape} {name}: {first_mismatch(got, ref)}"
        s.close()
    with pytest.raises(E.FlowLBError) as ei:  # the vector path takes at most 512 threads per CTA
        b.set_launch("team", 1, 2, 1024, vector=True)
    assert ei.value.status == 1
    b.close()


def _check_cases(b, ens, steps, bb=E.BB_HALFWAY, arith=E.ARITH_FUSED):
    for i, (flags, tau, gx, gy) in enumerate(ens):
        s = E.Solver(flags, precision=32, tau=tau, fx=gx, fy=gy, bounce_back=bb, arithmetic=arith)
        s.step(steps)
        for name, fid, ref in (("f", E.FIELD_F, s.f), ("rho", E.FIELD_RHO, s.rho), ("u", E.FIELD_U, s.u),
                               ("flags", E.FIELD_FLAGS, s.flags)):
            got = b.read(i, fid)
            assert exact_equal(got, ref), f"case {i} {flags.shape} {name}: {first_mismatch(got, ref)}"
        s.close()


@pytest.mark.parametrize("bb", [E.BB_HALFWAY, E.BB_IMPLICIT], ids=["halfway", "implicit"])
@pytest.mark.parametrize("arith", [E.ARITH_FUSED, E.ARITH_REFERENCE], ids=["fused", "ref-arith"])
def test_batch_streams_form_matches_single_handles(bb, arith):
    """The streams form (each case an engine handle, the cases' step graphs
    on concurrent streams): every case equals its own handle bit for bit,
    over launches of both parities, with more cases than streams."""
    ens = _small_ensemble(13, 1357)
    b = E.Batch(ens, bounce_back=bb, arithmetic=arith, autotune=0)
    b.set_launch("streams", 1, 4, 0)
    info = b.info()
    assert info["mode"] == "streams" and info["groups"] == 4
    for n in (2, 37, 27):
        b.step(n)
    b.sync()
    assert b.info()["t"] == 66
    _check_cases(b, ens, 66, bb, arith)
    b.close()


def test_batch_streams_form_switches_keep_the_state():
    """The state moves between the persistent kernel's arrays and the
    streams form's handles: the form is refused at an odd step, entered at
    an even one, left for a team shape, entered again; a reset in the form
    restarts every case; every case still equals its own handle."""
    ens = _small_ensemble(9, 2468)
    b = E.Batch(ens, autotune=0)
    b.set_launch("team", 2, 3, 256)
    b.step(3)
    with pytest.raises(E.FlowLBError) as ei:  # odd step: refused, the state stays in the batch's arrays
        b.set_launch("streams", 1, 3, 0)
    assert ei.value.status == 4
    b.step(1)
    b.set_launch("streams", 1, 3, 0)
    b.step(5)
    b.set_launch("team", 3, 2, 512)
    b.step(7)
    b.set_launch("streams", 1, 5, 0)
    b.step(4)
    b.sync()
    assert b.info()["t"] == 20
    _check_cases(b, ens, 20)
    b.reset()
    assert b.info()["t"] == 0 and b.info()["mode"] == "streams"
    b.step(6)
    b.sync()
    _check_cases(b, ens, 6)
    b.close()


def test_batch_tune_restricted_to_a_form():
    """flb_batch_tune among the streams form only and among the persistent
    kernel's shapes only: each keeps a shape of its form and restarts from
    the initial state."""
    ens = _small_ensemble(11, 97)
    b = E.Batch(ens, autotune=0)
    b.step(3)
    b.tune(8, E.TUNE_STREAMS)
    info = b.info()
    assert info["mode"] == "streams" and info["t"] == 0 and info["tuned"]
    b.step(10)
    b.tune(8, E.TUNE_PERSISTENT)
    info = b.info()
    assert info["mode"] in ("team", "cluster") and info["t"] == 0
    b.step(12)
    b.sync()
    _check_cases(b, ens, 12)
    with pytest.raises(E.FlowLBError):
        b.tune(8, 0)
    b.close()


def test_batch_rejects_unsupported_cases():
    ens = _small_ensemble(2, 1)
    with pytest.raises(E.FlowLBError):
        E.Batch(ens, bounce_back=E.BB_HALFWAY, arithmetic=7)


def test_batch_launch_shape_changes_keep_the_state():
    """flb_batch_set_launch between launches, clusters and teams: the cases
    still end equal to their own handles, whatever shape ran each part."""
    ens = _small_ensemble(11, 7)
    b = E.Batch(ens, autotune=0)
    steps = 0
    shapes = ((("cluster", 1, 5, 256), 3), (("team", 3, 4, 512, True), 6), (("cluster", 16, 1, 1024), 8),
              (("team", 1, 11, 256), 1), (("cluster", 4, 2, 256, True), 2), (("team", 7, 2, 1024), 5),
              (("cluster", 4, 3, 1024), 1))
    for shape, n in shapes:
        b.set_launch(*shape)
        info = b.info()
        assert (info["mode"], info["group"], info["groups"], info["threads"]) == shape[:4]
        assert info["vector"] == (len(shape) > 4)
        b.step(n)
        steps += n
    b.sync()
    assert b.info()["t"] == steps
    for i, (flags, tau, gx, gy) in enumerate(ens):
        s = E.Solver(flags, precision=32, tau=tau, fx=gx, fy=gy)
        s.step(steps)
        for fid, ref in ((E.FIELD_F, s.f), (E.FIELD_U, s.u)):
            got = b.read(i, fid)
            assert exact_equal(got, ref), f"case {i}: {first_mismatch(got, ref)}"
        s.close()
    for bad in (("cluster", 3, 1, 512), ("cluster", 8, 1, 384), ("cluster", 8, 0, 512), ("cluster", 8, 12, 512),
                ("team", 0, 2, 512)):
        with pytest.raises(E.FlowLBError) as ei:
            b.set_launch(*bad)
        assert ei.value.status == 1  # FLB_ERR_INVALID_ARGUMENT
    with pytest.raises(E.FlowLBError) as ei:  # more CTAs than fit on the device at once
        b.set_launch("team", 100000, 1, 1024)
    assert ei.value.status == 4  # FLB_ERR_UNSUPPORTED
    info = b.info()
    assert (info["mode"], info["group"], info["groups"], info["threads"]) == ("cluster", 4, 3, 1024)
    b.close()


def test_full_ensemble_matches_single_handles_at_5000_steps():
    """The 512-case culvert ensemble at its full sizes (nx up to 1024, ny up
    to 256) for its full 5,000 steps in the tuned launch shape: eight cases
    (the largest, the smallest and six seeded picks) equal their own handles
    bit for bit."""
    ens = cases.ensemble()
    b = E.Batch([(e.flags, e.tau, e.fx, 0.0) for e in ens], autotune=1)
    b.step(5000)
    b.sync()
    assert b.info()["t"] == 5000
    sizes = np.array([e.cells for e in ens])
    rng = np.random.default_rng(5000)
    picks = [int(sizes.argmax()), int(sizes.argmin())] + [int(k) for k in rng.choice(len(ens), 6, replace=False)]
    for i in picks:
        e = ens[i]
        s = E.Solver(e.flags, precision=32, tau=e.tau, fx=e.fx)
        s.step(5000)
        for name, fid, ref in (("f", E.FIELD_F, s.f), ("rho", E.FIELD_RHO, s.rho), ("u", E.FIELD_U, s.u),
                               ("flags", E.FIELD_FLAGS, s.flags)):
            got = b.read(i, fid)
            assert exact_equal(got, ref), f"case {i} {e.flags.shape} {name}: {first_mismatch(got, ref)}"
        s.close()
    b.close()


def test_team_barrier_wait_runs_out_and_reset_recovers(monkeypatch):
    """Failure detection of the team barrier, made on the host: with
    FLB_BATCH_SKIP_ARRIVAL=1 one CTA of every team never arrives, so every
    wait runs out after a short limit (4,096 polls) and the kernel leaves.
    flb_batch_sync reports FLB_ERR_CUDA, stepping is refused until
    flb_batch_reset, and after the reset the batch steps bit-equal to one
    handle per case.  The reference has no failure handling here: its CUDA
    error check exits the process (src/cuda/cudaUtils.cuh:17-26)."""
    ens = _small_ensemble(6, 99)
    b = E.Batch(ens, autotune=0)
    b.set_launch("team", 2, 3, 256)
    b.set_wait_limit(4096)
    monkeypatch.setenv("FLB_BATCH_SKIP_ARRIVAL", "1")
    b.step(9)
    with pytest.raises(E.FlowLBError) as ei:
        b.sync()
    assert ei.value.status == 2  # FLB_ERR_CUDA
    with pytest.raises(E.FlowLBError) as ei:
        b.step(1)
    assert ei.value.status == 2
    monkeypatch.delenv("FLB_BATCH_SKIP_ARRIVAL")
    b.reset()
    b.set_wait_limit(0)
    b.step(21)
    b.sync()
    assert b.info()["t"] == 21
    for i, (flags, tau, gx, gy) in enumerate(ens):
        s = E.Solver(flags, precision=32, tau=tau, fx=gx, fy=gy)
        s.step(21)
        got = b.read(i, E.FIELD_F)
        assert exact_equal(got, s.f), f"case {i}: {first_mismatch(got, s.f)}"
        s.close()
    b.close()
