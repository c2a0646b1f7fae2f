"""CPU tests of the file-based set-up (Geometry.txt + OptionsCalc.txt) and of
the VTK writer: host code of the engine library, no device calls.

Pins: the reference's own mesh.vti files (tests/golden/setup/, made by
tests/golden/make_setup_fixtures.py) are reproduced byte for byte, by the
engine and by the oracle restatement (oracle/setup_oracle.py).  Then the
engine is compared with the oracle on seeded synthetic inputs that exercise
every shape, boundary and option the reader knows, and on the reader's error
paths (src/io/reader.cpp)."""
import ctypes
import gzip
import math
import os
import random
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, ROOT
from flowlb_b200 import engine as E
from oracle import setup_oracle as SO

SETUP = os.path.join(GOLDEN, "setup")
CASES = ["damBreak", "cavity", "Poiseuille_plano", "modulos"]
W, F, G, I, IN, OUT = SO.WALL, SO.FLUID, SO.GAS, SO.INTERFACE, SO.INLET, SO.OUTLET


def golden_bytes(case):
    return gzip.decompress(open(os.path.join(SETUP, case, "mesh.vti.gz"), "rb").read())


def golden_flags(case, nx, ny):
    text = golden_bytes(case).decode()
    body = text.split('format="ascii">\n', 1)[1].split("</DataArray>", 1)[0]
    return np.array([int(v) for v in body.split()], np.uint8).reshape(ny, nx)


def paths(case):
    d = os.path.join(SETUP, case)
    return os.path.join(d, "Geometry.txt"), os.path.join(d, "OptionsCalc.txt")


# ---- pins -------------------------------------------------------------------

@pytest.mark.parametrize("case", CASES)
def test_mesh_vti_matches_reference_bytes(case, tmp_path):
    """App::createDomain's mesh.vti, byte for byte (flags, header, number format)."""
    s = E.Setup(*paths(case), mesh_only=True)
    out = str(tmp_path / "mesh.vti")
    s.write_mesh_vti(out)
    assert open(out, "rb").read() == golden_bytes(case)


# The golden cases as the oracle's structured description (the values of the
# fixture files).
ORACLE_CASES = {
    "damBreak": dict(points=[(0, 0, 0), (1, 0, 0)], size=0.01, idx_init=0, idx_end=1,
                     cdws=[dict(kind="CIRCLE", radius=0.5)],
                     obstacles=[dict(kind="RECT", x0=0.45, y0=0.05, z0=0.0, height=0.1, xwidth=0.05, zwidth=0.2,
                                     zrot=0.0)],
                     initial=[dict(kind="RECT", x0=0.2, y0=0.35, z0=0.0, height=0.5, xwidth=0.2, zwidth=0.2)],
                     free_surface=True, left=W, right=W, up=W, down=W),
    "cavity": dict(points=[(0, 0, 0), (0.1, 0, 0)], size=0.001, idx_init=0, idx_end=1,
                   cdws=[dict(kind="CIRCLE", radius=0.05)], free_surface=False, left=W, right=W, up=IN, down=W),
    "Poiseuille_plano": dict(points=[(0, 0, 0), (20, 0, 0)], size=0.005, idx_init=0, idx_end=1,
                             cdws=[dict(kind="CIRCLE", radius=0.1)], free_surface=False, left=IN, right=OUT,
                             up=W, down=W),
}


@pytest.mark.parametrize("case", sorted(ORACLE_CASES))
def test_oracle_reproduces_reference_mesh(case):
    c = ORACLE_CASES[case]
    m = SO.mesh_size(c)
    flags = SO.geometry_flags(c)
    if c["free_surface"]:
        flags = SO.free_surface_flags(flags)
    text = SO.vti_text([("Flags", "UInt8", flags, 1, 1.0, False)], m["nx"], m["ny"],
                       (m["xmin"], m["ymin"], m["zmin"]), m["size"])
    assert text == golden_bytes(case)


def test_dambreak_options_derive_reference_constants():
    """tau, force, inlet velocity and loop bounds of the damBreak inputs, as
    h_initConstantDataCuda2D and the headless loop compute them."""
    s = E.Setup(*paths("damBreak"))
    c = dict(ref_velocity_lb=0.1, ref_velocity_si=10.0, density=1000.0, nu=1.0e-6, use_force=True,
             acc=(0.0, -9.80665, 0.0), vforce=(0.0, 0.0, 0.0), velocity=(1.0, 0.0, 0.0), time_simulation=15.0,
             time_save=0.1)
    o = SO.derived(c, s.nx, 1.0)
    d = s.desc
    assert np.float32(d.tau) == o["tau"] and np.float32(d.fx) == o["fx"] and np.float32(d.fy) == o["fy"]
    assert d.inlet_ux == o["inlet_ux"] and d.inlet_uy == o["inlet_uy"]
    assert (s.time_steps, s.save_every) == (o["time_steps"], o["save_every"]) == (150000, 1000)
    assert d.free_surface == 1 and d.precision == 32 and d.mass_precision == 32 and d.subgrid == 1
    assert d.bounce_back == E.BB_IMPLICIT and d.fs_mode == E.FS_REFERENCE and d.arithmetic == E.ARITH_REFERENCE
    assert s.graphics_api == 1 and s.cuda_block == (16, 16, 0)


def test_structs_match_header():
    """Field offsets of flb_setup, flb_vti_field and flb_run_info against the
    ctypes mirrors."""
    specs = [("flb_setup", E.SetupStruct), ("flb_vti_field", E.VtiField), ("flb_run_info", E.RunInfo)]
    src = '#include <stdio.h>\n#include <stddef.h>\n#include "flowlb.h"\nint main(void){\n'
    for cname, st in specs:
        src += f'printf("{cname} size %zu\\n", sizeof({cname}));\n'
        for f, _ in st._fields_:
            src += f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "probe.c")
        exe = os.path.join(d, "probe")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out.strip().splitlines()}
    for cname, st in specs:
        assert got[(cname, "size")] == ctypes.sizeof(st), cname
        for f, _ in st._fields_:
            assert got[(cname, f)] == getattr(st, f).offset, (cname, f)


# ---- synthetic inputs: engine vs oracle -------------------------------------

BOUNDARY_NAMES = {IN: "INPUT", OUT: "OUTPUT", W: "WALL", F: "PERIODIC"}


def _r(rng, a, b, nd=3):
    return round(rng.uniform(a, b), nd)


def random_case(seed, directory):
    """A seeded description, the two files that hold it, and its CSV shapes."""
    rng = random.Random(seed)
    npts = rng.choice([2, 2, 3, 4])
    x = _r(rng, -2.0, 0.0, 2)
    pts = []
    y = 0.0
    for k in range(npts):
        pts.append((x, y, 0.0))
        x = round(x + _r(rng, 0.8, 2.0, 2), 2)
        y = round(y + _r(rng, -0.3, 0.3, 2), 2)
    if npts >= 3 and rng.random() < 0.4:
        idx_init, idx_end = 1, npts - 1
    else:
        idx_init, idx_end = 0, npts - 1
    length = pts[-1][0] - min(0.0, pts[0][0])
    size = round(length / rng.randint(40, 70), 4)
    cdws = []
    for _ in range(rng.choice([1, 1, 2])):
        if rng.random() < 0.8:
            cdws.append(dict(kind="CIRCLE", radius=_r(rng, 0.4, 1.0)))
        else:
            cdws.append(dict(kind="RECTANGLE", height=_r(rng, 0.8, 2.0)))
    xlo, xhi = min(0.0, pts[0][0]), pts[-1][0]
    obstacles, initial, csv = [], [], {}

    def polygon(name):
        n = rng.randint(3, 7)
        ang = sorted(rng.uniform(0, 2 * math.pi) for _ in range(n))
        rad = [_r(rng, 0.1, 0.4) for _ in range(n)]
        xs = [round(1.0 + r * math.cos(a), 4) for r, a in zip(rad, ang)]
        ys = [round(2.0 + r * math.sin(a), 4) for r, a in zip(rad, ang)]
        csv[name] = (xs, ys)
        return xs, ys

    for k in range(rng.randint(0, 3)):
        kind = rng.choice(["WALL", "CIRCLE", "CSV_2D"])
        x0, y0 = _r(rng, xlo + 0.2, xhi - 0.2), _r(rng, 0.1, 1.2)
        if kind == "WALL":
            obstacles.append(dict(kind="RECT", x0=x0, y0=y0, z0=0.0, height=_r(rng, 0.1, 0.6),
                                  xwidth=_r(rng, 0.05, 0.4), zwidth=0.2, zrot_deg=rng.choice([0, 0, 30, -45, 10])))
        elif kind == "CIRCLE":
            obstacles.append(dict(kind="CIRCLE", x0=x0, y0=y0, radius=_r(rng, 0.05, 0.3)))
        else:
            xs, ys = polygon(f"obst{k}")
            obstacles.append(dict(kind="POLY", x0=x0, y0=y0, xs=xs, ys=ys, name=f"obst{k}",
                                  zrot_deg=rng.choice([0, 20, -60])))
    fs = rng.random() < 0.5
    if fs:
        for k in range(rng.randint(1, 2)):
            x0, y0 = _r(rng, xlo + 0.3, xhi - 0.3), _r(rng, 0.3, 0.8)
            if rng.random() < 0.7:
                initial.append(dict(kind="RECT", x0=x0, y0=y0, z0=0.0, height=_r(rng, 0.2, 0.6),
                                    xwidth=_r(rng, 0.2, 0.8), zwidth=0.2))
            else:
                xs, ys = polygon(f"init{k}")
                initial.append(dict(kind="POLY", x0=x0, y0=y0, xs=xs, ys=ys, name=f"init{k}", zrot_deg=0))
    left = rng.choice([IN, W, OUT, F])
    right = left if left in (OUT, F) else rng.choice([IN, W, OUT, F])
    up, down = rng.choice([W, IN, OUT, F]), rng.choice([W, W, IN])
    opts = dict(ref_velocity_lb=rng.choice([0.05, 0.1]), ref_velocity_si=rng.choice([1.0, 2.0, 10.0]),
                density=rng.choice([1.0, 1000.0, 1.225]), nu=rng.choice([1e-6, 1e-3, 0.02]),
                use_force=rng.random() < 0.7, acc=(0.0, rng.choice([0.0, -9.80665]), 0.0),
                vforce=(rng.choice([0.0, 0.4]), 0.0, 0.0), velocity=(rng.choice([0.5, 1.0]), 0.0, 0.0),
                time_simulation=rng.choice([2.0, 3.5]), time_save=rng.choice([0.25, 0.5]),
                relaxation_time=rng.choice([0.0, 0.0, 0.6]))
    if opts["use_force"] and opts["acc"][1] == 0.0 and opts["vforce"][0] == 0.0:
        opts["vforce"] = (0.4, 0.0, 0.0)
    case = dict(points=pts, size=size, idx_init=idx_init, idx_end=idx_end, cdws=cdws, obstacles=[], initial=[],
                free_surface=fs, left=left, right=right, up=up, down=down, **opts)
    for o in obstacles:
        o2 = {k: v for k, v in o.items() if k not in ("zrot_deg", "name")}
        if "zrot_deg" in o:
            o2["zrot"] = o["zrot_deg"] * math.pi / 180.0
        case["obstacles"].append(o2)
    for o in initial:
        o2 = {k: v for k, v in o.items() if k not in ("zrot_deg", "name")}
        case["initial"].append(o2)

    g = ["# synthetic culvert", "TYPE_DOMAIN = 2D"]
    for k, p in enumerate(pts):
        g.append(f"POINT({k + 1}) = ({p[0]!r}, {p[1]!r}, {p[2]!r})")
    g += [f"SIZE = {size!r}", f"INITIAL_POSITION_SHAPES = {idx_init + 1}", f"END_POSITION_SHAPES = {idx_end + 1}"]
    for k, c in enumerate(cdws):
        g.append(f"CDW({k + 1}).type = {c['kind']}")
        if c["kind"] == "CIRCLE":
            g.append(f"CDW({k + 1}).radius = {c['radius']!r}")
        else:
            g.append(f"CDW({k + 1}).height = {c['height']!r}   # in y")
    g.append("SEPARATION = 2")
    for k, o in enumerate(obstacles):
        n = k + 1
        kind = {"RECT": "WALL", "CIRCLE": "CIRCLE", "POLY": "CSV_2D"}[o["kind"]]
        g.append(f"OBSTACLE({n}).type = {kind}")
        if o["kind"] == "POLY":
            g.append(f"OBSTACLE({n}).name = {o['name']}  # without .csv")
        g.append(f"OBSTACLE({n}).position = ({o['x0']!r}, {o['y0']!r}, 0)")
        if o["kind"] == "RECT":
            g += [f"OBSTACLE({n}).height = {o['height']!r}", f"OBSTACLE({n}).xWidth = {o['xwidth']!r}",
                  f"OBSTACLE({n}).zWidth = {o['zwidth']!r}"]
        if o["kind"] == "CIRCLE":
            g.append(f"OBSTACLE({n}).radius = {o['radius']!r}")
        if "zrot_deg" in o:
            g.append(f"OBSTACLE({n}).rotation = (0, 0, {o['zrot_deg']})")
    opt = ["TYPE_ANALYSIS = 2D", "CALCULATION_API = CUDA", "CUDA_BLOCK_SIZE = (16, 16, 1)", "GRAPHICS_API = NONE",
           f"TYPE_PROBLEM = {'FREE_SURFACE' if fs else 'MONOFLUID'}",
           f"USE_VOLUMETRIC_FORCE = {'TRUE' if opts['use_force'] else 'FALSE'}",
           "ACCELERATION = (%r, %r, 0) // y positive upwards" % opts["acc"][:2],
           "VOLUMETRIC_FORCE = (%r, 0, 0)" % opts["vforce"][0], "COLLISION_OPERATOR = SRT",
           "SUBGRID_TURBULENCE_MODEL = FALSE", "SURFACE_TENSION = FALSE", "PRECISION = 32",
           f"REFERENCE_VELOCITY_LB = {opts['ref_velocity_lb']!r}",
           f"REFERENCE_VELOCITY_SI = {opts['ref_velocity_si']!r} # m/s",
           "VELOCITY = (%r, 0, 0)" % opts["velocity"][0], f"KINEMATIC_VISCOSITY = {opts['nu']!r}",
           f"DENSITY = {opts['density']!r}"]
    if opts["relaxation_time"]:
        opt.append(f"RELAXATION_TIME = {opts['relaxation_time']!r}")
    opt += [f"LEFT_BOUNDARY = {BOUNDARY_NAMES[left]}", f"RIGHT_BOUNDARY = {BOUNDARY_NAMES[right]}",
            f"UP_BOUNDARY = {BOUNDARY_NAMES[up]}", f"DOWN_BOUNDARY = {BOUNDARY_NAMES[down]}"]
    for k, o in enumerate(initial):
        n = k + 1
        opt.append(f"INITIAL_CONDITION_FLAG({n}).type = {'CUBE' if o['kind'] == 'RECT' else 'CSV_2D'}")
        if o["kind"] == "POLY":
            opt.append(f"INITIAL_CONDITION_FLAG({n}).name = {o['name']}")
        opt.append(f"INITIAL_CONDITION_FLAG({n}).position = ({o['x0']!r}, {o['y0']!r}, 0)")
        if o["kind"] == "RECT":
            opt += [f"INITIAL_CONDITION_FLAG({n}).height = {o['height']!r}",
                    f"INITIAL_CONDITION_FLAG({n}).xWidth = {o['xwidth']!r}",
                    f"INITIAL_CONDITION_FLAG({n}).zWidth = {o['zwidth']!r}"]
    opt += [f"TIME_SIMULATION = {opts['time_simulation']!r}", f"TIME_SAVE = {opts['time_save']!r}"]
    gp, op = os.path.join(directory, "Geometry.txt"), os.path.join(directory, "OptionsCalc.txt")
    open(gp, "w").write("\n".join(g) + "\n")
    open(op, "w").write("\n\n".join(opt) + "\n")
    for name, (xs, ys) in csv.items():
        with open(os.path.join(directory, name + ".csv"), "w") as f:
            f.write("\n".join(f"{a!r};{b!r}" for a, b in zip(xs, ys)) + "\n")
    return case, gp, op


@pytest.mark.parametrize("seed", range(12))
def test_synthetic_inputs_match_oracle(seed, tmp_path):
    case, gp, op = random_case(seed, str(tmp_path))
    s = E.Setup(gp, op)
    m = SO.mesh_size(case)
    assert (s.nx, s.ny) == (m["nx"], m["ny"])
    assert s.origin == (m["xmin"], m["ymin"], m["zmin"]) and s.spacing == case["size"]
    want = SO.geometry_flags(case)
    np.testing.assert_array_equal(s.flags, want)
    want_init = SO.free_surface_flags(want) if case["free_surface"] else want
    np.testing.assert_array_equal(s.initial_flags, want_init)
    o = SO.derived(case, s.nx, m["xmax"] - m["xmin"])
    d = s.desc
    assert np.float32(d.tau) == o["tau"] and np.float32(d.fx) == o["fx"] and np.float32(d.fy) == o["fy"]
    assert d.inlet_ux == o["inlet_ux"] and d.inlet_uy == o["inlet_uy"]
    assert np.float32(s.nu_lattice) == o["nu"]
    assert (s.time_steps, s.save_every) == (o["time_steps"], o["save_every"])
    assert s.units["velocity"] == o["velocity"] and s.units["rho"] == o["rho"]
    assert d.free_surface == int(case["free_surface"])


def test_synthetic_inputs_cover_the_branches(tmp_path):
    """The seeds above reach every shape kind, every boundary type, the
    free-surface sweep, rotations and a CDW range narrower than the domain."""
    seen = set()
    for seed in range(12):
        case, _, _ = random_case(seed, str(tmp_path))
        seen |= {o["kind"] for o in case["obstacles"]} | {"init_" + o["kind"] for o in case["initial"]}
        seen |= {("b", case[k]) for k in ("left", "right", "up", "down")}
        seen |= {"fs"} if case["free_surface"] else {"mono"}
        seen |= {"rot"} if any(o.get("zrot", 0) for o in case["obstacles"]) else set()
        seen |= {"partial"} if case["idx_init"] > 0 else set()
        seen |= {c["kind"] for c in case["cdws"]}
    need = {"RECT", "CIRCLE", "POLY", "init_RECT", "fs", "mono", "rot", "partial", "RECTANGLE",
            ("b", IN), ("b", OUT), ("b", W), ("b", F)}
    assert need <= seen, need - seen


# ---- reader error paths -----------------------------------------------------

GEO_OK = """TYPE_DOMAIN = 2D
POINT(1) = (0, 0, 0)
POINT(2) = (1, 0, 0)
SIZE = 0.05
INITIAL_POSITION_SHAPES = 1
END_POSITION_SHAPES = 2
CDW(1).type = CIRCLE
CDW(1).radius = 0.25
"""
OPT_OK = """TYPE_ANALYSIS = 2D
CALCULATION_API = CUDA
CUDA_BLOCK_SIZE = (16,16,0)
GRAPHICS_API = NONE
TYPE_PROBLEM = MONOFLUID
USE_VOLUMETRIC_FORCE = TRUE
ACCELERATION = (0, 0, 0)
VOLUMETRIC_FORCE = (0.4,0,0)
COLLISION_OPERATOR = SRT
SUBGRID_TURBULENCE_MODEL = FALSE
PRECISION = 32
REFERENCE_VELOCITY_LB = 0.1
REFERENCE_VELOCITY_SI = 2.0
VELOCITY = (1, 0, 0)
KINEMATIC_VISCOSITY = 2e-3
DENSITY = 1
LEFT_BOUNDARY = INPUT
RIGHT_BOUNDARY = OUTPUT
UP_BOUNDARY = WALL
DOWN_BOUNDARY = WALL
TIME_SIMULATION = 3
TIME_SAVE = 1
"""


def _setup(tmp_path, geo=GEO_OK, opt=OPT_OK, mesh_only=False):
    gp, op = tmp_path / "Geometry.txt", tmp_path / "OptionsCalc.txt"
    gp.write_text(geo)
    op.write_text(opt)
    return E.Setup(str(gp), str(op), mesh_only=mesh_only)


def test_minimal_files_read(tmp_path):
    s = _setup(tmp_path)
    assert (s.nx, s.ny) == (21, 11)
    assert (s.flags[1:-1, 0] == IN).all() and (s.flags[1:-1, -1] == OUT).all()
    assert (s.flags[0] == W).all() and (s.flags[-1] == W).all() and (s.flags[1:-1, 1:-1] == F).all()


@pytest.mark.parametrize("geo_edit,opt_edit,status,message", [
    (None, ("UP_BOUNDARY = WALL", "UP_BOUNDARY = NOTHING"), 1, "UP_BOUNDARY cannot be NONE"),
    (None, ("LEFT_BOUNDARY = INPUT", "LEFT_BOUNDARY = PERIODIC"), 1, "must be equal if a periodic"),
    (None, ("TIME_SAVE = 1", "TIME_SAVE = 5"), 1, "The save time is greater than the simulation time, 5.0000 > 3.0000"),
    (None, ("TIME_SAVE = 1", "TIME_SAVE = 0"), 1, "The save time cannot be 0"),
    (None, ("DENSITY = 1", "DENSITY = 0"), 1, "The density has to have a value or be positive"),
    (None, ("KINEMATIC_VISCOSITY = 2e-3", "KINEMATIC_VISCOSITY = abc"), 1,
     "The value of the kinematic viscosity in the calculation's file in the line 15 is invalid"),
    (None, ("PRECISION = 32", "PRECISION = 8"), 1,
     "The value of the option in the calculation's file in the line 11 doesn't exist"),
    (None, ("PRECISION = 32", "PRECISIO = 32"), 1, "The option in the calculation's file in the line 11 doesn't exist"),
    (None, ("VELOCITY = (1, 0, 0)", "VELOCITY = (-1, 0, 0)"), 1, "cannot be negative"),
    (None, ("VELOCITY = (1, 0, 0)", "VELOCITY = (0, 0, 0)"), 1, "One of the two arguments, flow or velocity"),
    (None, ("CUDA_BLOCK_SIZE = (16,16,0)", "CUDA_BLOCK_SIZE = (64,32,0)"), 1,
     "The threads per block is superior to the maximum, 2048 > 1024"),
    (None, ("VOLUMETRIC_FORCE = (0.4,0,0)", "VOLUMETRIC_FORCE = (0,0,0)"), 1,
     "some values of the forces themselves or the acceleration must be indicated"),
    (None, ("TYPE_PROBLEM = MONOFLUID", "TYPE_PROBLEM = MONO = FLUID"), 1, "Error in the line 5"),
    (None, ("RELAXATION_TIME", "RELAXATION_TIME"), 0, None),
    (("POINT(2) = (1, 0, 0)", "POINT(1) = (1, 0, 0)"), None, 1, "maybe it is repeated"),
    (("END_POSITION_SHAPES = 2", "END_POSITION_SHAPES = 1"), None, 1, "cannot be equal or greater than the end"),
    (("INITIAL_POSITION_SHAPES = 1", "INITIAL_POSITION_SHAPES = 0"), None, 1, "it can't be the last point"),
    (("CDW(1).radius = 0.25", "CDW(2).radius = 0.25"), None, 1, "specify the type of CDW first"),
    (("CDW(1).type = CIRCLE", "CDW(1).type = SQUARE"), None, 1, "The shape of the CDW in the line 7 is not correct"),
    (("TYPE_DOMAIN = 2D", "TYPE_DOMAIN = 3D"), None, 4, "two-dimensional"),
])
def test_reader_errors(tmp_path, geo_edit, opt_edit, status, message):
    geo, opt = GEO_OK, OPT_OK
    if geo_edit:
        assert geo_edit[0] in geo
        geo = geo.replace(*geo_edit)
    if opt_edit:
        assert opt_edit[0] in opt or status == 0
        opt = opt.replace(*opt_edit)
    if status == 0:
        _setup(tmp_path, geo, opt)
        return
    with pytest.raises(E.FlowLBError) as ei:
        _setup(tmp_path, geo, opt)
    assert ei.value.status == status
    assert message in str(ei.value)


def test_missing_file_is_io_error(tmp_path):
    with pytest.raises(E.FlowLBError) as ei:
        E.Setup(str(tmp_path / "nope.txt"), str(tmp_path / "nope2.txt"))
    assert ei.value.status == 5


def test_reader_line_rules(tmp_path):
    """Comments, spaces inside values, trailing text after the third
    component and Windows line ends are read as FlowLB reads them; the
    mesh-only read ignores options it does not look for."""
    geo = GEO_OK.replace("SIZE = 0.05", "S I Z E = 0 . 05   # cell size").replace("\n", "\r\n")
    opt = OPT_OK.replace("VOLUMETRIC_FORCE = (0.4,0,0)", "VOLUMETRIC_FORCE = ( 0.4 , 0 , 0 ) // N/m3")
    s = _setup(tmp_path, geo, opt)
    assert (s.nx, s.ny) == (21, 11) and s.desc.fx > 0
    s2 = _setup(tmp_path, GEO_OK, OPT_OK.replace("PRECISION = 32", "PRECISION = 8"), mesh_only=True)
    assert (s2.flags == s.flags).all()


def test_unreached_nodes_keep_their_index_byte(tmp_path):
    """A node outside the CDW range and off the boundary rows keeps the low
    byte of its index (initData.h:261), as in the reference."""
    geo = GEO_OK.replace("POINT(2) = (1, 0, 0)", "POINT(2) = (0.5, 0, 0)\nPOINT(3) = (1, 0, 0)")
    s = _setup(tmp_path, geo)
    assert s.nx == 21
    y, x = 5, 15
    assert s.flags[y, x] == (x + y * s.nx) & 0xFF


# ---- VTK writer -------------------------------------------------------------

@pytest.mark.parametrize("seed", range(3))
def test_writer_matches_reference_format(seed, tmp_path):
    rng = np.random.default_rng(seed)
    nx, ny = 13, 7
    N = nx * ny
    flags = rng.integers(0, 256, N).astype(np.uint8)
    u32 = (rng.standard_normal(2 * N) * 10.0 ** rng.integers(-9, 4, 2 * N)).astype(np.float32)
    u32[:4] = [np.nan, np.inf, -0.0, 1e-40]
    r64 = 1.0 + rng.standard_normal(N) * 1e-3
    v3 = rng.standard_normal(3 * N)
    fields = [("Flags", flags, 1, 1.0, False), ("U", u32, 2, 100.0, seed == 1), ("rho", r64, 1, 1000.0, False),
              ("W", v3, 3, 0.5, True)]
    origin, spacing = (-4.8, 0.25, 0.0), 0.005
    out = str(tmp_path / "r.vti")
    E.write_vti(out, fields, nx, ny, origin, spacing)
    names = {np.dtype(np.uint8): "UInt8", np.dtype(np.float32): "Float32", np.dtype(np.float64): "Float64"}
    want = SO.vti_text([(n, names[a.dtype], a, c, k, fl) for n, a, c, k, fl in fields], nx, ny, origin, spacing)
    assert open(out, "rb").read() == want


def test_series_file(tmp_path):
    L = E.load_library()
    assert L.flb_write_vti_series(str(tmp_path).encode(), 3, 0.1) == 0
    assert (tmp_path / "loaderFiles.vti.series").read_bytes() == SO.series_text(3, 0.1)


def _reformat(text, rng):
    """The same file with whitespace inserted at random places (inside
    keywords and numbers too), '#' comments after some lines, comment-only
    lines between them and Windows line ends on some: every one of these is
    removed by FlowLB's line rules before a line is read."""
    out = []
    for line in text.splitlines():
        chars = list(line)
        for _ in range(int(rng.integers(0, 4))):
            chars.insert(int(rng.integers(0, len(chars) + 1)), str(rng.choice([" ", "  ", "\t"])))
        line = "".join(chars)
        if rng.random() < 0.3:
            line += " # note = (1, 2, 3)"
        if rng.random() < 0.2:
            out.append("# a comment line")
        out.append(line + ("\r" if rng.random() < 0.3 else ""))
    return "\n".join(out) + "\n"


@pytest.mark.parametrize("seed", range(8))
def test_reader_ignores_formatting(tmp_path, seed):
    """Seeded reformatting of valid input files (whitespace, comments, line
    ends) gives the same lattice, flags, constants and loop bounds."""
    base = _setup(tmp_path, GEO_OK, OPT_OK)
    rng = np.random.default_rng(1000 + seed)
    d = tmp_path / "fmt"
    d.mkdir()
    s = _setup(d, _reformat(GEO_OK, rng), _reformat(OPT_OK, rng))
    assert (s.nx, s.ny) == (base.nx, base.ny)
    assert (s.flags == base.flags).all() and (s.initial_flags == base.initial_flags).all()
    for f in ("tau", "fx", "fy", "inlet_ux", "inlet_uy", "free_surface", "precision"):
        assert getattr(s.desc, f) == getattr(base.desc, f), f
    assert (s.time_steps, s.save_every, s.cuda_block) == (base.time_steps, base.save_every, base.cuda_block)


def test_reader_comment_rule_removes_spaces_only(tmp_path):
    """FlowLB skips a line when, after removing spaces (' ' only), it is
    empty or starts with '#' (reader.cpp:720-723).  A comment indented by a
    tab, or a blank line that holds only a carriage return, therefore reaches
    the option parser as an empty option: the options reader rejects it as an
    unknown option (reader.cpp:543-547), the geometry reader ignores it.  The
    engine keeps both behaviours."""
    for extra in ("\t# indented by a tab", "\r"):
        opt = OPT_OK.replace("GRAPHICS_API = NONE", "GRAPHICS_API = NONE\n" + extra)
        with pytest.raises(E.FlowLBError) as ei:
            _setup(tmp_path, GEO_OK, opt)
        assert ei.value.status == 1
        assert "The option in the calculation's file in the line 5 doesn't exist" in str(ei.value)
        geo = GEO_OK.replace("SIZE = 0.05", "SIZE = 0.05\n" + extra)
        s = _setup(tmp_path, geo, OPT_OK)
        assert (s.nx, s.ny) == (21, 11)
    # indented by spaces, the same comment is skipped
    _setup(tmp_path, GEO_OK, OPT_OK.replace("GRAPHICS_API = NONE", "GRAPHICS_API = NONE\n    # spaces"))
