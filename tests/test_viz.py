"""Headless visualisation: CPU checks of the oracle restatement
(oracle/viz_oracle.py) and GPU parity of the engine's k_viz.cu kernels with
it, bit for bit, on fields read back from real runs."""
import math

import numpy as np
import pytest

from flowlb_b200 import cases
from flowlb_b200 import engine as E
from oracle import viz_oracle as VO


# ---- CPU: the oracle on analytic inputs --------------------------------------

def test_mirrored_repeat_lookup():
    """A 4-entry ramp: s = 0.5 lands between texels 1 and 2; s = 1.25 wraps
    back (mirrored); s = -0.3 clamps to 0 (GLSL max)."""
    cmap = np.array([[0, 0, 0], [0.25, 0, 0], [0.5, 0, 0], [1.0, 0, 0]], np.float32)
    u = np.array([0.5, 1.25, -0.3, 0.125, 0, 0, 0, 0], np.float32)  # ux of 4 nodes, then uy
    rgba = VO.shade(u, VO.UX, cmap, 1.0, 0.0)
    # s=0.5: coord 1.5 -> texels 1,2, a=0.5 -> 0.375
    assert rgba[0, 0] == round(0.375 * 255)
    # s=1.25: coord 4.5 -> texels 4,5 wrap to 3,2, a=0.5 -> 0.75
    assert rgba[1, 0] == round(0.75 * 255)
    # s=0 (clamped): coord -0.5 -> texels -1,0 wrap to 0,0 -> 0
    assert rgba[2, 0] == 0
    # s=0.125: coord 0 -> texels 0,1, a=0 -> 0
    assert rgba[3, 0] == 0
    assert (rgba[:, 3] == 255).all()


def test_isoline_of_a_circle_is_a_closed_ring():
    nx = ny = 48
    y, x = np.mgrid[0:ny, 0:nx]
    r = np.hypot(x - 23.5, y - 23.5).astype(np.float32)
    u = np.concatenate([r.ravel(), np.zeros(nx * ny, np.float32)])
    img = VO.isoline(u, nx, ny, True, 15.0, nx, ny, (0, nx, 0, ny))
    on = np.argwhere(img == 255)
    assert len(on) > 2 * math.pi * 15 * 0.8
    dist = np.hypot(on[:, 1] - 23.5, on[:, 0] - 23.5)
    assert np.all(np.abs(dist - 15.0) < 2.0)


# ---- GPU: engine kernels vs the oracle ---------------------------------------

def _state(precision, steps=60):
    case = cases.small_dam_break(96, 64)
    s = E.Solver(case.flags, free_surface=True, precision=precision, mass_precision=64, tau=case.tau,
                 fx=case.fx, fy=case.fy, bounce_back=E.BB_HALFWAY, fs_mode=E.FS_CONSERVATIVE, u_max=0.25)
    s.step(steps)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [32, 64])
def test_viz_kernels_match_oracle(require_gpu, precision):
    s = _state(precision)
    try:
        u = s.read(E.FIELD_U)
        phi = s.read(E.FIELD_PHI)
        img = s.viz_velocity()
        np.testing.assert_array_equal(img.reshape(-1, 2), VO.velocity_image(u))
        rng = np.random.default_rng(7)
        cmap = np.sort(rng.random((256, 3)).astype(np.float32), axis=0)
        mag = np.hypot(u[:s.N], u[s.N:])
        vmax = float(np.percentile(mag, 99))
        for q, (hi, lo) in [(E.VIZ_UX, (vmax, -vmax)), (E.VIZ_UY, (vmax, -vmax)), (E.VIZ_MAGNITUDE, (vmax, 0.0)),
                            (E.VIZ_PRESSURE, (0.5 * vmax, 0.01))]:
            got = s.viz_shade(q, cmap, hi, lo)
            want = VO.shade(u, q, cmap, hi, lo)
            np.testing.assert_array_equal(got.reshape(-1, 4), want, err_msg=f"quantity {q}")
        iso_u = float(np.percentile(mag[mag > 0], 60))
        for field, iso, vec in [(E.FIELD_U, iso_u, True), (E.FIELD_PHI, 0.5, False)]:
            src = u if vec else phi
            for (w, h, b) in [(s.nx, s.ny, (0, s.nx, 0, s.ny)), (2 * s.nx, 2 * s.ny, (0, s.nx, 0, s.ny)),
                              (301, 157, (10, 70, 5, 50))]:
                got = s.viz_isoline(field, iso, w, h, b)
                want = VO.isoline(src, s.nx, s.ny, vec, iso, w, h, b)
                assert (want == 255).sum() > 20
                np.testing.assert_array_equal(got, want, err_msg=f"field {field} {w}x{h} {b}")
    finally:
        s.close()


@pytest.mark.gpu
def test_viz_rejects_bad_arguments(require_gpu):
    s = _state(32, steps=2)
    try:
        with pytest.raises(E.FlowLBError):
            s.viz_shade(7, np.zeros((4, 3), np.float32), 1.0, 0.0)
        with pytest.raises(E.FlowLBError):
            s.viz_isoline(E.FIELD_RHO, 0.5, 10, 10)
        with pytest.raises(E.FlowLBError):
            s.viz_isoline(E.FIELD_U, 0.5, 10, 10, (5, 5, 0, 10))
        with pytest.raises(E.FlowLBError):
            s.viz_isoline(E.FIELD_U, 0.5, 10, 10, (0, s.nx + 1, 0, 10))
    finally:
        s.close()
