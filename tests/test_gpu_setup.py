"""GPU tests of the file-based path: ``flb_create_from_files`` builds the
initial state FlowLB builds from its example inputs, and
``flb_run_from_files`` writes the result files FlowLB's headless loop writes,
byte for byte against the oracle stepped from the same set-up.

The engine runs in the reference's modes here (IMPLICIT walls, REFERENCE free
surface and arithmetic, the PRECISION of the options file), which the oracle
reproduces bit for bit, so the written text must be identical."""
import gzip
import os

import numpy as np
import pytest

from conftest import GOLDEN
from flowlb_b200 import engine as E
from oracle import oracle as O
from oracle import setup_oracle as SO

pytestmark = pytest.mark.gpu
SETUP = os.path.join(GOLDEN, "setup")


def golden_flags(case, nx, ny):
    text = gzip.decompress(open(os.path.join(SETUP, case, "mesh.vti.gz"), "rb").read()).decode()
    body = text.split('format="ascii">\n', 1)[1].split("</DataArray>", 1)[0]
    return np.array([int(v) for v in body.split()], np.uint8).reshape(ny, nx)


def paths(case, directory=SETUP):
    d = os.path.join(directory, case)
    return os.path.join(d, "Geometry.txt"), os.path.join(d, "OptionsCalc.txt")


@pytest.mark.parametrize("case", ["damBreak", "Poiseuille_plano", "modulos"])
def test_create_from_files_builds_reference_initial_flags(require_gpu, case):
    s = E.Solver.from_files(*paths(case))
    try:
        flags = s.read(E.FIELD_FLAGS).reshape(s.ny, s.nx)
        np.testing.assert_array_equal(flags, golden_flags(case, s.nx, s.ny))
        rho = s.read(E.FIELD_RHO)
        solid = (flags.ravel() & (SO.WALL | SO.GAS)) != 0
        assert np.all(rho[~solid] == 1.0)
    finally:
        s.close()


def test_create_from_files_rejects_an_inlet_in_the_last_cell(require_gpu):
    """The cavity's lid is an INLET row that ends in the last cell, whose
    inlet rule reads the density one cell past the end of the lattice
    (lbmKernel2D.cu:334-340); creation refuses it before allocating."""
    with pytest.raises(E.FlowLBError) as ei:
        E.Solver.from_files(*paths("cavity"))
    assert ei.value.status == 1


def _short_run_inputs(tmp_path, case, time_simulation, time_save):
    geo, opt = paths(case)
    d = tmp_path / case
    d.mkdir()
    (d / "Geometry.txt").write_text(open(geo).read())
    lines = []
    for line in open(opt).read().splitlines():
        key = line.split("=")[0].strip()
        if key == "TIME_SIMULATION":
            line = f"TIME_SIMULATION = {time_simulation}"
        elif key == "TIME_SAVE":
            line = f"TIME_SAVE = {time_save}"
        elif key == "GRAPHICS_API":
            line = "GRAPHICS_API = NONE"
        lines.append(line)
    (d / "OptionsCalc.txt").write_text("\n".join(lines) + "\n")
    return str(d / "Geometry.txt"), str(d / "OptionsCalc.txt")


def _oracle_for(setup):
    d = setup.desc
    variant = {64: O.F64, 32: O.F32_M32 if d.mass_precision == 32 else O.F32}[d.precision]
    cfg = O.OracleConfig(variant=variant, free_surface=bool(d.free_surface), bb=O.BB_IMPLICIT,
                         fs_mode=O.FS_REFERENCE, collision=d.collision, subgrid=bool(d.subgrid),
                         use_force=bool(d.use_volumetric_force), tau=d.tau, fx=d.fx, fy=d.fy,
                         inlet_ux=d.inlet_ux, inlet_uy=d.inlet_uy, arithmetic=O.ARITH_REFERENCE)
    return O.Oracle(setup.flags, cfg)


# (case, TIME_SIMULATION, TIME_SAVE): 12 and 5 lattice steps for both (T = 1e-4 s
# for damBreak, 2.5e-4 s for the channel), so 13 steps and saves after steps 0,
# 5 and 10.
RUNS = [("damBreak", 0.0012, 0.0005), ("Poiseuille_plano", 0.003, 0.00125)]


@pytest.mark.parametrize("case,t_sim,t_save", RUNS)
def test_run_from_files_writes_reference_results(require_gpu, tmp_path, case, t_sim, t_save):
    geo, opt = _short_run_inputs(tmp_path, case, t_sim, t_save)
    setup = E.Setup(geo, opt)
    assert (setup.time_steps, setup.save_every) == (12, 5)
    out = tmp_path / "out"
    out.mkdir()
    info = E.run_from_files(geo, opt, str(out))
    assert info["steps"] == 13 and info["files"] == 3
    assert info["directory"].endswith("results_0")
    o = _oracle_for(setup)
    fs = bool(setup.desc.free_surface)
    typ = "Float64" if setup.desc.precision == 64 else "Float32"
    uc = 1.0 if fs else setup.units["velocity"]
    rc = 1.0 if fs else setup.units["rho"]
    done = 0
    for k, t_save_step in enumerate([0, 5, 10]):
        o.step(t_save_step + 1 - done)
        done = t_save_step + 1
        fields = [("Flags", "UInt8", o.flags, 1, 1.0, False), ("U", typ, o.u, 2, uc, False),
                  ("rho", typ, o.rho, 1, rc, False)]
        if fs:
            fields.append(("phi", typ, o.phi, 1, 1.0, False))
        want = SO.vti_text(fields, setup.nx, setup.ny, setup.origin, setup.spacing)
        got = open(os.path.join(info["directory"], f"result_{k}.vti"), "rb").read()
        assert got == want, f"result_{k}.vti differs from the oracle"
    series = open(os.path.join(info["directory"], "loaderFiles.vti.series"), "rb").read()
    assert series == SO.series_text(3, float(np.float32(t_save)))
    # a second run goes to a new folder, as the reference's writer does
    info2 = E.run_from_files(geo, opt, str(out), max_steps=1)
    assert info2["directory"].endswith("results_1") and info2["files"] == 1 and info2["steps"] == 1
