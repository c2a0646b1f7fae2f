"""CPU restatement of FlowLB's geometry stage, unit conversion and VTK writer.

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of the engine's
file-based set-up (``flb_setup_from_files``) and VTK writer
(``flb_write_vti``).  The engine never imports it.

Pinned by the reference's own mesh.vti files (tests/golden/setup/): the
flags and the writer output of this module and of the engine are both
compared with them byte for byte.

It works on a structured description of the inputs (the values the two
files hold), not on the files, so that a test can write the files from the
same description and check the engine's parser and geometry together:

    case = dict(points=[(x, y, z), ...], size=..., idx_init=0, idx_end=1,
                cdws=[dict(kind="CIRCLE", radius=r) | dict(kind="RECTANGLE", height=h)],
                obstacles=[shape, ...], initial=[shape, ...],
                free_surface=bool, left=.., right=.., up=.., down=..)
    shape = dict(kind="RECT", x0, y0, z0, height, xwidth, zwidth, zrot)
          | dict(kind="CIRCLE", x0, y0, radius)
          | dict(kind="POLY", x0, y0, zrot, xs=[...], ys=[...])

Reference files followed: src/initData.h:42-66 and 220-317 (flag sweep),
src/initData.cpp:13-124 (free-surface sweep), src/geometry/shapes.cpp
(shape tests), src/math/math.cpp:89-103 (point-line distance),
src/geometry/mesh.cpp:44-51 (lattice size), src/io/reader.cpp:1126-1156
(domain height from the CDWs), src/utils.cpp:7-82 and
src/cuda/cudaInitData.cu:57-82 (units, tau, force), src/io/writer.cpp
(VTK text).  Pure Python loops: use small grids.
"""
from __future__ import annotations

import math

import numpy as np

FLUID, GAS, INTERFACE, WALL, INLET, OUTLET = 0x01, 0x02, 0x04, 0x08, 0x20, 0x40
EPS = 1e-12


def mesh_size(case: dict) -> dict:
    """Bounding box (starting at the origin), domain height from the CDWs and
    the lattice size (Mesh::calculateNumberPointsMesh)."""
    xmin = xmax = ymin = ymax = zmin = zmax = 0.0
    for (x, y, z) in case["points"]:
        if x > xmax:
            xmax = x
        if x < xmin:
            xmin = x
        if y > ymax:
            ymax = y
        if y < ymin:
            ymin = y
        if z > zmax:
            zmax = z
        if z < zmin:
            zmin = z
    pts = case["points"]
    h0, h1 = pts[case["idx_init"]][1], pts[case["idx_end"]][1]
    for c in case["cdws"]:
        add = 2 * c["radius"] if c["kind"] == "CIRCLE" else c["height"]
        a, b = h0 + add, h1 + add
        if a > ymax:
            ymax = a
        if b > ymax:
            ymax = b
    size = case["size"]
    nx = int(math.floor((xmax - xmin) / size) + 1)
    ny = int(math.floor((ymax - ymin) / size) + 1)
    return dict(xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax, zmin=zmin, zmax=zmax, nx=nx, ny=ny, size=size)


def _prepare(shape: dict) -> dict:
    s = dict(shape)
    if s["kind"] == "RECT":
        z = s.get("zrot", 0.0)
        s["rotate"] = not (abs(z - 0.0) <= 1e-6)
        s["rx"] = (math.cos(-z), math.sin(-z))
        s["ry"] = (math.sin(-z), math.cos(-z))
        x0, y0, z0 = s["x0"], s["y0"], s.get("z0", 0.0)
        s["box"] = (x0 - s["xwidth"] / 2.0 - EPS, x0 + s["xwidth"] / 2.0 + EPS,
                    y0 - s["height"] / 2.0 - EPS, y0 + s["height"] / 2.0 + EPS,
                    z0 - s.get("zwidth", 0.0) / 2.0 - EPS, z0 + s.get("zwidth", 0.0) / 2.0 + EPS)
    elif s["kind"] == "POLY":
        xs, ys = list(map(float, s["xs"])), list(map(float, s["ys"]))
        n = len(xs)
        area = cx = cy = 0.0
        for i in range(n - 1):
            p = xs[i] * ys[i + 1] - xs[i + 1] * ys[i]
            area += p
            cx += (xs[i] + xs[i + 1]) * p
            cy += (ys[i] + ys[i + 1]) * p
        p = (xs[n - 1] * ys[0] - xs[0] * ys[n - 1])
        area += p
        cx += (xs[n - 1] + xs[0]) * p
        cy += (ys[n - 1] + ys[0]) * p
        area *= 0.5
        area = -area if area < 0 else area
        cx /= (6.0 * area)
        cx = -cx if cx < 0 else cx
        cy /= (6.0 * area)
        cy = -cy if cy < 0 else cy
        z = s.get("zrot", 0.0)
        rot = not (abs(z - 0.0) <= 1e-6)
        c, sn = math.cos(z), math.sin(z)
        bx0 = bx1 = by0 = by1 = 0.0
        for i in range(n):
            x, y = xs[i] - cx, ys[i] - cy
            if rot:
                prev = x
                x = x * c - y * sn
                y = prev * sn + y * c
            x += s["x0"]
            y += s["y0"]
            xs[i], ys[i] = x, y
            if x > bx1:
                bx1 = x
            elif x < bx0:
                bx0 = x
            if y > by1:
                by1 = y
            elif y < by0:
                by0 = y
        s["pxs"], s["pys"] = xs, ys
        s["box"] = (bx0 - EPS, bx1 + EPS, by0 - EPS, by1 + EPS)
    return s


def _inside(s: dict, x: float, y: float, z: float) -> bool:
    k = s["kind"]
    if k == "CIRCLE":
        d2 = (y - s["y0"]) * (y - s["y0"]) + (x - s["x0"]) * (x - s["x0"])
        return not (d2 > (s["radius"] * s["radius"] + EPS))
    if k == "RECT":
        if s["rotate"]:
            px, py = x - s["x0"], y - s["y0"]
            x = px * s["rx"][0] - py * s["rx"][1]
            y = px * s["ry"][0] + py * s["ry"][1]
            x += s["x0"]
            y += s["y0"]
        b = s["box"]
        return not (x > b[1] or x < b[0] or y > b[3] or y < b[2] or z > b[5] or z < b[4])
    b = s["box"]
    if x > b[1] or x < b[0] or y > b[3] or y < b[2]:
        return False
    xs, ys = s["pxs"], s["pys"]
    inside = False
    j = len(xs) - 1
    for i in range(len(xs)):
        if ((ys[i] > y) != (ys[j] > y)) and (x < (xs[j] - xs[i]) * (y - ys[i]) / (ys[j] - ys[i]) + xs[i]):
            inside = not inside
        j = i
    return inside


def _cdw_inside(c: dict, x, y, z, p, b) -> bool:
    if c["kind"] == "CIRCLE":
        r = c["radius"]
        qx, qy, qz = x - p[b][0], y - (p[b][1] + r), z - p[b][2]
        vx, vy, vz = p[b - 1][0] - p[b][0], p[b - 1][1] - p[b][1], p[b - 1][2] - p[b][2]
        cx, cy, cz = qy * vz - qz * vy, qz * vx - qx * vz, qx * vy - qy * vx
        d2 = (cx * cx + cy * cy + cz * cz) / (vx * vx + vy * vy + vz * vz)
        return d2 <= (r * r + EPS)
    slope = (p[b][1] - p[b - 1][1]) / (p[b][0] - p[b - 1][0])
    ydown = p[b - 1][1] + (x - p[b - 1][0]) * slope
    return (y >= (ydown - EPS)) and (y <= (ydown + EPS))


def geometry_flags(case: dict) -> np.ndarray:
    """The (ny, nx) flags of initData's first sweep."""
    m = mesh_size(case)
    p = [tuple(map(float, q)) for q in case["points"]]
    obstacles = [_prepare(s) for s in case.get("obstacles", [])]
    initial = [_prepare(s) for s in case.get("initial", [])]
    dflt = GAS if case["free_surface"] else FLUID
    ix, ex = p[case["idx_init"]][0] - EPS, p[case["idx_end"]][0] + EPS
    nx, ny, size = m["nx"], m["ny"], m["size"]
    out = np.zeros((ny, nx), np.uint8)
    for y in range(ny):
        for x in range(nx):
            idx = x + y * nx
            f = idx & 0xFF
            xs, ys, zs = m["xmin"] + x * size, m["ymin"] + y * size, m["zmin"] + 0 * size
            b = len(p) - 1
            for k in range(1, len(p)):
                if p[k][0] >= xs - 1e-12:
                    b = k
                    break
            slope = (p[b][1] - p[b - 1][1]) / (p[b][0] - p[b - 1][0])
            base = p[b - 1][1] + (xs - p[b - 1][0]) * slope
            if xs >= ix and xs <= ex:
                for c in case["cdws"]:
                    f = dflt if _cdw_inside(c, xs, ys, zs, p, b) else WALL
            else:
                if ys <= base + EPS:
                    f = case["down"]
                elif ys >= m["ymax"] - EPS:
                    f = case["up"]
            if ys <= base + EPS and f == dflt:
                f = case["down"]
            elif ys >= m["ymax"] - EPS and f == dflt:
                f = case["up"]
            elif x == 0 and f == dflt:
                f = case["left"]
            elif x == nx - 1 and f == dflt:
                f = case["right"]
            for s in obstacles:
                if _inside(s, xs, ys, zs):
                    f = WALL
            for s in initial:
                if _inside(s, xs, ys, zs):
                    f = FLUID
            out[y, x] = f
    return out


def free_surface_flags(flags: np.ndarray) -> np.ndarray:
    """initFreeSurfaceFlags over every cell in index order."""
    f = flags.copy()
    ny, nx = f.shape
    for y in range(ny):
        for x in range(nx):
            v = int(f[y, x])
            if v & ~(FLUID | INLET | OUTLET) & 0xFF:
                continue
            if v & INLET:
                v |= FLUID
            elif v & OUTLET:
                v |= GAS
            f[y, x] = v
            if not v & FLUID:
                continue
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if (dx or dy) and 0 <= x + dx < nx and 0 <= y + dy < ny and f[y + dy, x + dx] == GAS:
                        f[y + dy, x + dx] = INTERFACE
    return f


def derived(case: dict, nx: int, length: float) -> dict:
    """Units, tau, body force (float) and loop bounds, in the reference's
    operation order and types."""
    L = length / float(nx - 1)
    T = L * case["ref_velocity_lb"] / case["ref_velocity_si"]
    M = case["density"] / 1.0 * (L * L * L)
    f32 = np.float32
    if not (abs(case.get("relaxation_time", 0.0) - 0.0) <= 1e-6):
        nu = f32((case["relaxation_time"] - 0.5) / 3.0)
        tau = f32(case["relaxation_time"])
    else:
        nu = f32(float(f32(case["nu"])) * T / (L * L))
        tau = f32(f32(3.0) * nu + f32(0.5))

    def force(acc, vf):
        if abs(acc - 0.0) <= 1e-6:
            return f32(vf * T * T * L * L / M)
        return f32(case["density"] * acc * L * L * T * T / M)

    fx = fy = f32(0.0)
    if case.get("use_force", False):
        fx = force(case["acc"][0], case["vforce"][0])
        fy = force(case["acc"][1], case["vforce"][1])
    steps = lambda t: int(f32(float(f32(t)) / T))
    return dict(L=L, T=T, M=M, nu=nu, tau=tau, fx=fx, fy=fy, velocity=L / T, rho=M / (L * L * L),
                inlet_ux=case["velocity"][0] / (L / T), inlet_uy=case["velocity"][1] / (L / T),
                time_steps=steps(case["time_simulation"]), save_every=steps(case["time_save"]))


def vti_text(fields, nx: int, ny: int, origin=(0.0, 0.0, 0.0), spacing: float = 1.0) -> bytes:
    """VTIWriter output (writer.cpp:15-60, 214-252): values as %g, origin and
    spacing as %f.  ``fields``: (name, vtk type, array, components, to_si, flip_y)."""
    ext = f"0 {nx - 1} 0 {ny - 1} 0 0"
    sp = f"{spacing:f}"
    out = ['<VTKFile type="ImageData" version="1.0">\n',
           f'<ImageData WholeExtent="{ext}" Origin="{origin[0]:f} {origin[1]:f} {origin[2]:f}" '
           f'Spacing="{sp} {sp} {sp}" >\n', f'<Piece Extent="{ext}" >\n', "<PointData>\n"]
    N = nx * ny
    for name, vtype, arr, comps, to_si, flip in fields:
        a = np.asarray(arr).ravel()
        out.append(f'<DataArray type="{vtype}" Name="{name}" NumberOfComponents="{comps}" format="ascii">\n')
        vals = [float(v) for v in a.tolist()]
        sgn = -1.0 if flip else 1.0
        for i in range(N):
            if comps == 1:
                out.append("%g\n" % (vals[i] * to_si))
            else:
                line = "%g %g" % (vals[i] * to_si, vals[i + N] * to_si * sgn)
                if comps == 3:
                    line += " %g" % (vals[i + 2 * N] * to_si)
                out.append(line + "\n")
        out.append("</DataArray>\n")
    out.append("</PointData>\n<CellData>\n</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n")
    return "".join(out).encode()


def series_text(n_files: int, dt: float) -> bytes:
    s = '{\n"file-series-version" : "1.0",\n"files" : [\n'
    for i in range(n_files):
        s += '{"name" : "result_%d.vti", "time" : %f},\n' % (i, i * dt)
    return (s + "]\n}").encode()
