"""The FP64 CPU tape adjoint (oracle/flb_adjoint_oracle.c) against central
finite differences of its own forward model (CPU only)."""
import numpy as np

from flowlb_b200 import cases
from oracle import oracle as O


def test_tape_adjoint_matches_central_differences():
    c = cases.porous_channel(40, 12)
    s = c.porosity.astype(np.float64)
    steps, window, tau, gx = 160, 40, 0.6, 5e-6
    J, ds, dg = O.adjoint_run(c.flags, s, tau, gx, 0.0, steps, window)
    assert J > 0
    rng = np.random.default_rng(11)
    cells = np.argwhere((c.flags == cases.FLUID) & (s > 2e-3) & (s < 1 - 2e-3))
    eps = 1e-3
    for k in rng.choice(len(cells), 6, replace=False):
        y, x = cells[k]
        sp, sm = s.copy(), s.copy()
        sp[y, x] += eps
        sm[y, x] -= eps
        Jp = O.adjoint_run(c.flags, sp, tau, gx, 0.0, steps, window, grad=False)[0]
        Jm = O.adjoint_run(c.flags, sm, tau, gx, 0.0, steps, window, grad=False)[0]
        fd = (Jp - Jm) / (2 * eps)
        assert abs(fd - ds[y, x]) <= 1e-5 * abs(fd), (y, x, fd, ds[y, x])
    h = gx * 1e-4
    Jp = O.adjoint_run(c.flags, s, tau, gx + h, 0.0, steps, window, grad=False)[0]
    Jm = O.adjoint_run(c.flags, s, tau, gx - h, 0.0, steps, window, grad=False)[0]
    fd = (Jp - Jm) / (2 * h)
    assert abs(fd - dg[0]) <= 1e-6 * abs(fd), (fd, dg)
