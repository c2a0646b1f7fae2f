"""The engine's adjoint (flb_adjoint_*) against the FP64 CPU tape adjoint
and against central finite differences of its own FP64 forward."""
import numpy as np
import pytest

from flowlb_b200 import cases
from flowlb_b200 import engine as E
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("K", [2, 16, 64], ids=lambda k: f"ckpt{k}")
def test_fp64_adjoint_equals_cpu_tape(K):
    """Same formulas and operand order: J and dJ/ds bit for bit, dJ/dg to
    summation order (the engine sums per block, the tape cell by cell)."""
    c = cases.porous_channel(48, 16)
    s = c.porosity.astype(np.float64)
    steps, window = 256, 64
    a = E.Adjoint(c.flags, s, tau=0.6, gx=5e-6, precision=64, steps=steps, window=window, checkpoint_every=K)
    J = a.forward()
    ds, dg = a.backward()
    J0, ds0, dg0 = O.adjoint_run(c.flags, s, 0.6, 5e-6, 0.0, steps, window)
    assert J == J0
    assert np.array_equal(ds, ds0)
    assert np.allclose(dg, dg0, rtol=1e-12, atol=0)
    # a second backward (same forward) gives the same result
    ds2, dg2 = a.backward()
    assert np.array_equal(ds, ds2) and np.array_equal(dg, dg2)
    a.close()


def test_fp32_adjoint_close_to_fp64():
    """FP32 storage and arithmetic: the drag keeps u ~ 1e-5 while f ~ 0.1, so
    single precision resolves u to ~1e-3 relative; J and the gradient are held
    to 1e-2."""
    c = cases.porous_channel(128, 32)
    s = c.porosity.astype(np.float64)
    kw = dict(tau=0.6, gx=5e-6, steps=512, window=128, checkpoint_every=64)
    a64 = E.Adjoint(c.flags, s, precision=64, **kw)
    a32 = E.Adjoint(c.flags, s, precision=32, **kw)
    J64, J32 = a64.forward(), a32.forward()
    ds64, dg64 = a64.backward()
    ds32, dg32 = a32.backward()
    assert abs(J32 - J64) <= 1e-2 * abs(J64)
    fl = c.flags == cases.FLUID
    rel = np.linalg.norm(ds32[fl] - ds64[fl]) / np.linalg.norm(ds64[fl])
    assert rel < 1e-2, rel
    assert abs(dg32[0] - dg64[0]) <= 1e-2 * abs(dg64[0])
    a64.close()
    a32.close()


def test_adjoint_matches_finite_differences_full_case():
    """The porous culvert case at its full size (1024x256, 4096 steps, the
    last 512 in the objective, checkpoints every 64): the FP64 adjoint
    against central differences (eps = 1e-3) on 32 seeded cells and on g_x;
    relative agreement 1e-4 is required.  The cells are drawn among those
    whose |dJ/ds| is at least 1 % of the largest: J carries rounding of
    ~1e-13 relative, so a difference quotient with eps = 1e-3 cannot resolve
    gradients much below 1e-10 (far upstream cells reach 1e-13, where the
    quotient is rounding noise)."""
    c = cases.porous_channel()
    s = c.porosity.astype(np.float64)
    a = E.Adjoint(c.flags, s, tau=0.6, gx=5e-6, precision=64, steps=4096, window=512, checkpoint_every=64)
    a.forward()
    ds, dg = a.backward()
    rng = np.random.default_rng(11)
    eps = 1e-3
    big = np.abs(ds) >= 1e-2 * np.abs(ds).max()
    cand = np.argwhere((c.flags == cases.FLUID) & (s > eps) & (s < 1 - eps) & big)
    worst = 0.0
    for k in rng.choice(len(cand), 32, replace=False):
        y, x = cand[k]
        sp, sm = s.copy(), s.copy()
        sp[y, x] += eps
        sm[y, x] -= eps
        a.set_porosity(sp)
        Jp = a.forward()
        a.set_porosity(sm)
        Jm = a.forward()
        fd = (Jp - Jm) / (2 * eps)
        worst = max(worst, abs(fd - ds[y, x]) / abs(fd))
    a.set_porosity(s)
    h = 5e-6 * 1e-3
    a.set_force(5e-6 + h)
    Jp = a.forward()
    a.set_force(5e-6 - h)
    Jm = a.forward()
    fdg = (Jp - Jm) / (2 * h)
    print(f"worst relative FD error over 32 cells: {worst:.2e}; dJ/dgx {dg[0]:.6e} vs FD {fdg:.6e}")
    assert worst <= 1e-4
    assert abs(fdg - dg[0]) <= 1e-4 * abs(fdg)
    a.close()


def test_fp64_adjoint_cost_within_three_forwards():
    """The FP64 form, whose gradient meets the finite-difference check above on
    the same full-size case (1024x256, 4096 steps, checkpoints every 64), costs
    at most three forward passes: backward (recomputation included) over
    forward, device time of each, best of three after a warm-up pair."""
    c = cases.porous_channel()
    a = E.Adjoint(c.flags, c.porosity.astype(np.float64), tau=0.6, gx=5e-6, precision=64, steps=4096,
                  window=512, checkpoint_every=64)
    a.forward()
    a.backward()
    ratios = []
    for _ in range(3):
        a.forward()
        a.backward()
        f_ms, b_ms = a.timing()
        ratios.append(b_ms / f_ms)
    a.close()
    print(f"FP64 backward / forward: {min(ratios):.3f} (runs {', '.join(f'{r:.3f}' for r in ratios)})")
    assert min(ratios) <= 3.0, ratios
