"""The engine against its CPU twin on the benchmark configurations at their
stated sizes and lengths (through the C ABI).

The FP32 engine and the FP32 oracle round every operation alike, so the
populations, flags and FP64 free-surface fields must stay equal bit for bit
for the whole run, not only on the short small-grid runs of
test_gpu_engine.py: a single threshold that flips differently (an interface
conversion, a fill-level clamp) would show here as a first divergence step.

* the 256x64 culvert channel: single phase, g_x = 1e-6, tau = 0.6, 10,000
  steps, FP32 storage, in the engine's modes (half-way walls, fused
  arithmetic) and in the reference's (implicit walls, reference arithmetic);
* the 2048x512 free-surface dam break: FP32 populations, FP64 mass,
  tau = 0.55, g_y = -5e-5, half-way walls, conservative free surface,
  velocity limiter 0.25, fused arithmetic, 20,000 steps (the reference loop,
  src/cuda/runCuda.cu:493-528, runs kernels lbmKernel2D.cu:14-303 per step).
"""
import os

import numpy as np
import pytest

from conftest import exact_equal, first_mismatch
from flowlb_b200 import cases
from flowlb_b200 import engine as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _compare(s, o, fs):
    """Names of the fields that differ, with their first mismatch."""
    pairs = [("f", s.f, o.f64().astype(np.float32)), ("rho", s.rho, o.rho), ("u", s.u, o.u),
             ("flags", s.flags, o.flags)]
    if fs:
        pairs += [("mass", s.mass, o.mass), ("excess", s.excess, o.excess), ("phi", s.phi, o.phi)]
    return {name: first_mismatch(a, b) for name, a, b in pairs if not exact_equal(a, b)}


def _twin_run(s, o, fs, total, every):
    """Steps both by `every` up to `total`, comparing after each chunk; fails
    with the first chunk end at which any field differs."""
    t = 0
    while t < total:
        n = min(every, total - t)
        s.step(n)
        o.step(n)
        t += n
        bad = _compare(s, o, fs)
        assert not bad, f"first divergence by step {t} (checked every {every}): {bad}"
    assert s.t == o.t == total


@pytest.mark.parametrize("modes", ["engine", "reference"])
def test_channel_256x64_fp32_10000_steps_equals_oracle(modes):
    c = cases.plain_channel()
    assert (c.nx, c.ny, c.fx, c.tau) == (256, 64, 1e-6, 0.6)
    if modes == "engine":
        bb, arith = O.BB_HALFWAY, O.ARITH_FUSED
    else:
        bb, arith = O.BB_IMPLICIT, O.ARITH_REFERENCE
    s = E.Solver(c.flags, precision=32, tau=c.tau, fx=c.fx, bounce_back=bb, arithmetic=arith)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32, bb=bb, tau=c.tau, fx=c.fx, threads=THREADS,
                                         arithmetic=arith))
    _twin_run(s, o, False, 10_000, 1000)
    assert exact_equal(s.flags, c.flags.ravel())
    # the flow is developing: the channel core moves
    fl = np.tile(c.flags.ravel() == cases.FLUID, 2)
    assert np.abs(s.u[fl]).max() > 1e-5
    s.close()
    o.close()


def test_dam_break_2048x512_20000_steps_equals_oracle():
    c = cases.dam_break(1)
    kw = dict(tau=c.tau, fy=c.fy, u_max=0.25)
    s = E.Solver(c.flags, free_surface=True, precision=32, mass_precision=64, bounce_back=E.BB_HALFWAY,
                 fs_mode=E.FS_CONSERVATIVE, arithmetic=E.ARITH_FUSED, **kw)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32, free_surface=True, bb=O.BB_HALFWAY,
                                         fs_mode=O.FS_CONSERVATIVE, arithmetic=O.ARITH_FUSED, threads=THREADS,
                                         **kw))
    m0 = o.total_mass()
    _twin_run(s, o, True, 20_000, 1000)
    # FP64 mass conserved to round-off, on both sides
    assert abs(o.total_mass() - m0) / m0 < 1e-6
    assert abs(s.total_mass() - o.total_mass()) <= 1e-12 * m0  # same fields, different summation order
    cnt = s.cell_counts()
    assert cnt["fluid"] > 0 and cnt["interface"] > 0
    s.close()
    o.close()
