"""CPU tests of the oracle: pinned to the reference's own code and to known answers."""
import glob
import os

import numpy as np
import pytest

from conftest import GOLDEN, exact_equal
from flowlb_b200 import cases
from oracle import oracle as O

VARIANT_OF_PREC = {32: O.F32_M32, 64: O.F64}


def _init_fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "init_*.npz")))


@pytest.mark.parametrize("path", _init_fixtures(), ids=lambda p: os.path.basename(p))
def test_oracle_init_matches_reference_fixture(path):
    """Initial state equals FlowLB's own initFields/initFreeSurface* output."""
    g = dict(np.load(path))
    prec = 32 if "_p32" in path else 64
    fs = "dambreak" in path
    o = O.Oracle(g["geometry"], O.OracleConfig(variant=VARIANT_OF_PREC[prec], free_surface=fs))
    for k in ("f", "rho", "u", "flags"):
        assert exact_equal(getattr(o, k), g[k]), k
    if fs:
        for k in ("mass", "phi", "excess"):
            assert exact_equal(getattr(o, k), g[k]), k


@pytest.mark.skipif(not O.ref_host_available(), reason="reference host library not built")
@pytest.mark.parametrize("name", ["channel", "dambreak2048"])
@pytest.mark.parametrize("prec", [32, 64])
def test_oracle_init_matches_reference_full_size(name, prec):
    case = cases.plain_channel() if name == "channel" else cases.dam_break(1)
    ref = O.ref_host_init(case.flags, prec, case.free_surface)
    o = O.Oracle(case.flags, O.OracleConfig(variant=VARIANT_OF_PREC[prec], free_surface=case.free_surface))
    for k in ("f", "rho", "u", "flags"):
        assert exact_equal(getattr(o, k), ref[k]), k
    if case.free_surface:
        for k in ("mass", "phi", "excess"):
            assert exact_equal(getattr(o, k), ref[k]), k


@pytest.mark.skipif(not O.ref_host_available(), reason="reference host library not built")
def test_oracle_init_inlet_outlet_matches_reference():
    """Inlet cells take the inlet velocity and the FLUID bit, outlet cells the GAS bit."""
    flags = cases.small_dam_break(40, 32).flags.copy()
    flags[5:20, 1] = cases.INLET
    flags[3:10, 38] = cases.OUTLET
    for prec in (32, 64):
        ref = O.ref_host_init(flags, prec, True, inlet_ux=0.05, inlet_uy=0.01)
        o = O.Oracle(flags, O.OracleConfig(variant=VARIANT_OF_PREC[prec], free_surface=True, inlet_ux=0.05,
                                           inlet_uy=0.01))
        for k in ("f", "rho", "u", "flags", "mass", "phi", "excess"):
            assert exact_equal(getattr(o, k), ref[k]), (prec, k)


def _step_fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "step_*.npz")))


@pytest.mark.parametrize("path", _step_fixtures(), ids=lambda p: os.path.basename(p))
def test_oracle_steps_match_reference_cuda_fixture(path):
    """Oracle (reference mode) after N steps equals FlowLB's CUDA kernels
    (--fmad=false) after N steps, recorded on a B200 by make_golden.py --cuda."""
    g = dict(np.load(path))
    prec = 32 if "_p32" in path else 64
    fs = "dambreak" in path
    cfg = O.OracleConfig(variant=VARIANT_OF_PREC[prec], free_surface=fs, tau=float(g["tau"]), fx=float(g["fx"]),
                         fy=float(g["fy"]))
    o = O.Oracle(g["geometry"], cfg)
    o.step(int(g["steps"]))
    for k in ("f", "rho", "u", "flags"):
        assert exact_equal(getattr(o, k), g[k]), k
    if fs:
        for k in ("mass", "phi", "excess"):
            assert exact_equal(getattr(o, k), g[k]), k


def _kernel_fixtures():
    return sorted(glob.glob(os.path.join(GOLDEN, "kernels_*.npz")))


@pytest.mark.parametrize("path", _kernel_fixtures(), ids=lambda p: os.path.basename(p))
def test_oracle_kernels_match_reference_cuda_fixture(path):
    """Along the oracle's dam-break trajectory, each of FlowLB's five CUDA
    kernels (recorded on a B200 by make_golden.py --cuda) and the oracle's
    kernel give the same fields; for the two kernels that race in the
    reference, each cell must match one of the two interleavings."""
    from refcheck import check_kernel, snapshot
    g = dict(np.load(path))
    prec = 32 if "_p32" in path else 64
    geo = g["geometry"]
    cfg = O.OracleConfig(variant=VARIANT_OF_PREC[prec], free_surface=True, tau=float(g["tau"]),
                         fx=float(g["fx"]), fy=float(g["fy"]))
    o = O.Oracle(geo, cfg)
    names = {O.K_FS1: "fs1", O.K_STREAM_COLLIDE: "sc", O.K_FS2: "fs2", O.K_FS3: "fs3", O.K_FS4: "fs4"}
    samples = set(int(s) for s in g["sample_steps"])
    checked = 0
    for step in range(max(samples) + 1):
        for kid in (O.K_FS1, O.K_STREAM_COLLIDE, O.K_FS2, O.K_FS3, O.K_FS4):
            if step in samples:
                prefix = f"s{step}_{names[kid]}_"
                ref = {k[len(prefix):]: v for k, v in g.items() if k.startswith(prefix)}
                check_kernel(geo, cfg, snapshot(o), o.t, kid, ref, f"step {step} {names[kid]}")
                checked += 1
            o.kernel(kid)
        o.t = o.t + 1
    assert checked == 5 * len(samples)


def test_oracle_poiseuille_halfway_known_answer():
    """Body-force channel with half-way walls converges to the analytic
    parabola u(y) = F/(2 nu) (y - 1/2)(H + 1/2 - y), walls half a cell outside
    the first and last fluid rows, nu = (tau - 1/2)/3."""
    nx, ny, tau, F = 4, 18, 0.9, 1e-5
    flags = np.full((ny, nx), cases.FLUID, np.uint8)
    flags[0, :] = cases.WALL
    flags[-1, :] = cases.WALL
    o = O.Oracle(flags, O.OracleConfig(variant=O.F64, tau=tau, fx=F, bb=O.BB_HALFWAY))
    o.step(8000)
    ux = o.u[: nx * ny].reshape(ny, nx)[1:-1, 1]
    nu = (tau - 0.5) / 3.0
    H = ny - 2
    y = np.arange(1, ny - 1) - 0.5
    exact = F / (2 * nu) * y * (H - y)
    err = np.linalg.norm(ux - exact) / np.linalg.norm(exact)
    assert err < 5e-3, err


def test_oracle_halfway_conserves_single_phase_mass():
    c = cases.plain_channel(64, 32)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F64, tau=c.tau, fx=1e-5, bb=O.BB_HALFWAY))
    m0 = o.total_mass()
    o.step(300)
    assert abs(o.total_mass() - m0) / m0 < 1e-12


def test_oracle_conservative_free_surface_conserves_mass_fp64():
    c = cases.small_dam_break(64, 48)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F64, free_surface=True, tau=c.tau, fy=c.fy, bb=O.BB_HALFWAY,
                                         fs_mode=O.FS_CONSERVATIVE))
    m0 = o.total_mass()
    for _ in range(4):
        o.step(150)
        assert abs(o.total_mass() - m0) / m0 < 1e-12
    fl = o.flags
    assert set(np.unique(fl)).issubset({cases.FLUID, cases.GAS, cases.INTERFACE, cases.WALL})


def test_oracle_fp32_dd_fp64_mass_conserves_to_1e6():
    c = cases.small_dam_break(64, 48)
    o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32, free_surface=True, tau=c.tau, fy=c.fy, bb=O.BB_HALFWAY,
                                         fs_mode=O.FS_CONSERVATIVE))
    m0 = o.total_mass()
    o.step(600)
    assert abs(o.total_mass() - m0) / m0 < 1e-6


def test_oracle_fp16s_close_to_fp64():
    c = cases.plain_channel(64, 32)
    outs = {}
    for var in (O.F64, O.F16S):
        o = O.Oracle(c.flags, O.OracleConfig(variant=var, tau=c.tau, fx=1e-5, bb=O.BB_HALFWAY))
        o.step(400)
        outs[var] = o.u.astype(np.float64)
    fluid = np.tile((c.flags.ravel() == cases.FLUID), 2)
    a, b = outs[O.F16S][fluid], outs[O.F64][fluid]
    assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-3


def test_oracle_fs_count_pre_post_only_differ_by_ig_neighbours():
    """Running FS_4 with pre- and post-conversion neighbour counts differs only
    in cells that have an interface->gas neighbour."""
    c = cases.small_dam_break(64, 48)
    res = {}
    for pre in (False, True):
        o = O.Oracle(c.flags, O.OracleConfig(variant=O.F64, free_surface=True, tau=c.tau, fy=c.fy,
                                             fs_count_pre=pre))
        o.step(40)
        for k in (O.K_FS1, O.K_STREAM_COLLIDE, O.K_FS2, O.K_FS3):
            o.kernel(k)
        flags3 = o.flags.copy()
        o.kernel(O.K_FS4)
        res[pre] = (flags3, o.excess.copy(), o.mass.copy())
    flags3 = res[False][0]
    assert exact_equal(flags3, res[True][0])
    diff = (res[False][1] != res[True][1]) | (res[False][2] != res[True][2])
    ig = (flags3 & 0x86) == 0x06
    ny, nx = c.flags.shape
    igm = ig.reshape(ny, nx)
    near = np.zeros_like(igm)
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            if dx or dy:
                near |= np.roll(np.roll(igm, dy, 0), dx, 1)
    assert not np.any(diff & ~near.ravel())


def test_oracle_deterministic():
    c = cases.small_dam_break(48, 40)
    outs = []
    for _ in range(2):
        o = O.Oracle(c.flags, O.OracleConfig(variant=O.F32, free_surface=True, tau=c.tau, fy=c.fy))
        o.step(100)
        outs.append((o.f.copy(), o.mass.copy(), o.flags.copy()))
    for a, b in zip(*outs):
        assert exact_equal(a, b)


def test_f16_stochastic_rounding_matches_recorded_instruction():
    """orc_f16_rs (the FP16S stores' rounding) against cvt.rs.f16x2.f32 as
    recorded on a B200 (tests/golden/f16_rs_probe.npz): binary16 normal,
    subnormal and near-maximum results."""
    import os

    import numpy as np

    from oracle import oracle as O
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "f16_rs_probe.npz"))
    L = O.lib()
    got = np.array([L.orc_f16_rs_pair(int(x), int(y), int(z)) for x, y, z in zip(d["a"], d["b"], d["r"])],
                   np.uint32)
    np.testing.assert_array_equal(got, d["out"])


def _random_free_surface_box(seed):
    """A walled box with 1-3 solid blocks on the floor, a water column on one
    side and a free drop of water above the floor, all seeded."""
    rng = np.random.default_rng(seed)
    nx, ny = int(rng.integers(40, 81)), int(rng.integers(32, 65))
    g = np.full((ny, nx), cases.GAS, np.uint8)
    for _ in range(int(rng.integers(1, 4))):
        w, h = int(rng.integers(2, nx // 4)), int(rng.integers(2, ny // 3))
        x0 = int(rng.integers(1, nx - w - 1))
        g[1:1 + h, x0:x0 + w] = cases.WALL
    cw, ch = int(rng.integers(4, nx // 2)), int(rng.integers(6, ny - 8))
    col = g[1:1 + ch, 1:1 + cw]
    col[col == cases.GAS] = cases.FLUID
    r = int(rng.integers(2, 6))
    cx, cy = int(rng.integers(cw + r + 3, nx - r - 2)), int(rng.integers(ny // 2, ny - r - 3))
    yy, xx = np.mgrid[0:ny, 0:nx]
    drop = ((xx - cx) ** 2 + (yy - cy) ** 2 <= r * r) & (g == cases.GAS)
    g[drop] = cases.FLUID
    g[0, :] = g[-1, :] = g[:, 0] = g[:, -1] = cases.WALL
    tau = float(rng.uniform(0.52, 0.8))
    return g, tau


@pytest.mark.parametrize("seed", range(6))
@pytest.mark.parametrize("mode", [(O.FS_CONSERVATIVE, O.BB_HALFWAY), (O.FS_REFERENCE, O.BB_IMPLICIT),
                                  (O.FS_REFERENCE, O.BB_HALFWAY)],
                         ids=["conservative-halfway", "reference-implicit", "reference-halfway"])
def test_oracle_free_surface_invariants_on_random_boxes(seed, mode):
    """FP64 free surface with gravity on seeded random geometries: every
    non-solid cell is exactly one of fluid, interface or gas, and no fluid cell
    touches a gas cell (the interface layer closes), in the reference's rules
    and in the conservative ones; with the conservative rules and half-way
    walls the total mass (fill plus pending excess) also stays constant to
    round-off (the reference's rules lose mass: about 5e-5 of it over these
    200 steps with its implicit walls)."""
    fs_mode, bb = mode
    g, tau = _random_free_surface_box(seed)
    o = O.Oracle(g, O.OracleConfig(variant=O.F64, free_surface=True, tau=tau, fy=-1e-4, bb=bb, fs_mode=fs_mode,
                                   u_max=0.25))
    m0 = o.total_mass()
    ny, nx = g.shape
    for _ in range(5):
        o.step(40)
        if fs_mode == O.FS_CONSERVATIVE:
            assert abs(o.total_mass() - m0) / m0 < 1e-12
        fl = o.flags.reshape(ny, nx)
        assert set(np.unique(fl)).issubset({cases.FLUID, cases.GAS, cases.INTERFACE, cases.WALL})
        fluid = fl == cases.FLUID
        gas = fl == cases.GAS
        near_gas = np.zeros_like(gas)
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                near_gas |= np.roll(np.roll(gas, dy, 0), dx, 1)
        assert not np.any(fluid & near_gas), np.argwhere(fluid & near_gas)[:5]
    assert np.all(np.isfinite(o.rho))
