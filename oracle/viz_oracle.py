"""CPU restatement of the headless visualisation kernels (k_viz.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/ as the checker of
``flb_viz_velocity``, ``flb_viz_shade`` and ``flb_viz_isoline``.

Follows, in float32 with one rounding per operation:
* save2DDataToOpenGL, src/cuda/cudaUtils.cu:107-118;
* the fragment stage of assets/shaders/*/texture*2D.glsl with OpenGL's 1D
  texture lookup (GL_LINEAR, GL_MIRRORED_REPEAT: OpenGL 4.5 §8.14.2, the
  texel wrap  i' = (n-1) - mirror((i mod 2n) - n)) and the UNORM8 conversion
  round(clamp(c, 0, 1) * 255);
* d_CreateIsoSurfaceVector2D / getInterpolatedPoint / drawLine /
  marchingSquares, src/cuda/cudaIsosurface.cuh:33-199 and
  cudaIsosurface.cu:16-76 (Bresenham after Zingl, "A Rasterizing Algorithm
  for Drawing Curves", 2016).
Magnitudes are sqrt(x*x + y*y) as the engine computes them.
"""
from __future__ import annotations

import numpy as np

f32 = np.float32
UX, UY, MAGNITUDE, PRESSURE = 0, 1, 2, 3


def velocity_image(u: np.ndarray) -> np.ndarray:
    N = u.size // 2
    return np.stack([u[:N].astype(f32), u[N:].astype(f32)], axis=1)


def _mag(x, y):
    x = np.asarray(x, f32)
    y = np.asarray(y, f32)
    return np.sqrt(x * x + y * y, dtype=f32)


def shade(u: np.ndarray, quantity: int, cmap: np.ndarray, vmax: float, vmin: float) -> np.ndarray:
    N = u.size // 2
    ux, uy = u[:N].astype(f32), u[N:].astype(f32)
    v = ux if quantity == UX else uy if quantity == UY else _mag(ux, uy)
    with np.errstate(all="ignore"):
        s = (v - f32(vmin)) / (f32(vmax) - f32(vmin))
    s = np.where(s < 0, f32(0), s).astype(f32)
    s = np.where(np.isnan(s), f32(0), s).astype(f32)
    s = np.minimum(s, f32(1024.0))
    n = cmap.shape[0]
    coord = s * f32(n) - f32(0.5)
    fl = np.floor(coord).astype(f32)
    a = (coord - fl).astype(f32)
    i0 = fl.astype(np.int64)
    two = 2 * n

    def wrap(i):
        j = i % two
        return np.where(j < n, j, two - 1 - j)

    c0, c1 = cmap[wrap(i0)].astype(f32), cmap[wrap(i0 + 1)].astype(f32)
    c = (f32(1.0) - a)[:, None] * c0 + a[:, None] * c1
    c = np.clip(c, f32(0), f32(1)).astype(f32)
    rgb = np.rint(c * f32(255.0)).astype(np.uint8)
    return np.concatenate([rgb, np.full((N, 1), 255, np.uint8)], axis=1)


def _interp(p0, p1, v0, v1, iso):
    aux = (iso - v0) / (v1 - v0)
    aux2 = f32(1.0) - aux
    return (aux2 * p0[0] + aux * p1[0], aux2 * p0[1] + aux * p1[1])


def _draw(img, p0, p1, ppn, xo, yo, width, height):
    xp0, xp1 = p0[0] + xo, p1[0] + xo
    yp0, yp1 = p0[1] + yo, p1[1] + yo
    fx0 = ppn[0] * xp0 - f32(1.0) * f32(int(xp0) != 0) + f32(0.5)
    fx1 = ppn[0] * xp1 - f32(1.0) * f32(int(xp1) != 0) + f32(0.5)
    fy0 = f32(height) - ppn[1] * yp0 - f32(0.5)
    fy1 = f32(height) - ppn[1] * yp1 - f32(0.5)
    lx, ly = f32(width) + f32(2.0), f32(height) + f32(2.0)
    if not (abs(fx0) <= lx and abs(fx1) <= lx and abs(fy0) <= ly and abs(fy1) <= ly):
        return
    x0, y0, x1, y1 = int(fx0), int(fy0), int(fx1), int(fy1)
    dx, dy = abs(x1 - x0), -abs(y1 - y0)
    err = dx + dy
    sx, sy = (1 if x0 < x1 else -1), (1 if y0 < y1 else -1)
    guard = dx - dy + 1
    while (x0 != x1 or y0 != y1) and guard > 0:
        if 0 <= x0 < width and 0 <= y0 < height:
            img[y0, x0] = 255
        e2 = 2 * err
        if e2 >= dy:
            err += dy
            x0 += sx
        if e2 <= dx:
            err += dx
            y0 += sy
        guard -= 1


EDGES = {1: [((0, 1), (0, 3))], 14: [((0, 1), (0, 3))], 2: [((0, 1), (1, 2))], 13: [((0, 1), (1, 2))],
         3: [((0, 3), (1, 2))], 12: [((0, 3), (1, 2))], 4: [((1, 2), (3, 2))], 11: [((1, 2), (3, 2))],
         5: [((0, 1), (0, 3)), ((3, 2), (1, 2))], 6: [((0, 1), (3, 2))], 9: [((0, 1), (3, 2))],
         7: [((0, 3), (3, 2))], 8: [((0, 3), (3, 2))], 10: [((0, 3), (3, 2)), ((0, 1), (1, 2))]}
P = [(f32(0), f32(0)), (f32(1), f32(0)), (f32(1), f32(1)), (f32(0), f32(1))]


def isoline(field: np.ndarray, nx: int, ny: int, vector: bool, iso: float, width: int, height: int,
            bounds) -> np.ndarray:
    """The uint8 (height, width) image of the iso-line value = iso."""
    N = nx * ny
    if vector:
        val = _mag(field[:N], field[N:2 * N])
    else:
        val = field[:N].astype(f32)
    iso = f32(iso)
    b0, b1, b2, b3 = (int(b) for b in bounds)
    img = np.zeros((height, width), np.uint8)
    ppn = (f32(width) / f32(b1 - b0), f32(height) / f32(b3 - b2))
    for y in range(max(b2, 0), min(b3, ny - 1)):
        r = ny - y - 1
        for x in range(max(b0, 0), min(b1, nx - 1)):
            idx = x + r * nx
            v = [val[idx], val[idx + 1], val[idx - nx + 1], val[idx - nx]]
            sq = int(v[0] > iso) | (int(v[1] > iso) << 1) | (int(v[2] > iso) << 2) | (int(v[3] > iso) << 3)
            if sq in (0, 15):
                continue
            xo, yo = f32(x - b0), f32(y - b2)
            with np.errstate(all="ignore"):
                for (a0, a1), (c0, c1) in EDGES[sq]:
                    p = _interp(P[a0], P[a1], v[a0], v[a1], iso)
                    q = _interp(P[c0], P[c1], v[c0], v[c1], iso)
                    _draw(img, p, q, ppn, xo, yo, width, height)
    return img
