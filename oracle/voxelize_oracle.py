"""CPU restatement of the reference's voxeliser -- TEST INFRASTRUCTURE ONLY.

Follows web/js/voxelize.js:5-115 of RICKxxROLLING/wind-tunnel line by line in Python floats
(IEEE double, as JavaScript Numbers are), with the reference's operation order:

  * ray parity along +x per (y, z) column with the ray jittered by (0.01373, 0.00717)
    (voxelize.js:9-49);
  * the surface shell, Math.round of sampled points (voxelize.js:51-71);
  * a flood fill of fluid from the boundary (voxelize.js:73-92);
  * frontal/planform areas, count, and the y = 0 ground layer (voxelize.js:94-115).

Stated differences: a triangle with a non-finite coordinate is skipped (the reference's loops
run zero times for NaN; for infinities its output depends on the sort order of NaN keys), and
`(ux - vx) ** 2` is taken as the product (ux - vx) * (ux - vx).

Parity unpinned: no JavaScript runtime is available to run the reference itself, so this
restatement is checked by analytic properties (tests/test_voxelize_oracle.py) and the CUDA
voxeliser is compared with it bit for bit.
"""
import math
from collections import deque

import numpy as np

OY, OZ = 0.01373, 0.00717  # voxelize.js:9


def _js_round(x):
    """Math.round: nearest integer, halves towards +infinity (voxelize.js:63-65)."""
    f = math.floor(x)
    return f + 1 if x - f >= 0.5 else f


def _finite(p):
    return all(math.isfinite(v) for v in p)


def voxelize(tris, nx, ny, nz, ground):
    """tris: (T, 9) float32 (lattice coordinates). Returns (solid uint8 (n,), frontal,
    planform, count) as voxelize.js returns them."""
    tris = np.asarray(tris, np.float32).reshape(-1, 9)
    n = nx * ny * nz
    vox = np.zeros(n, np.uint8)
    cols = {}
    for t in range(len(tris)):
        p = [float(v) for v in tris[t]]
        if not _finite(p):
            continue
        ax, ay, az, bx, by, bz, cx, cy, cz = p
        y0 = max(1, math.ceil(min(ay, by, cy) - OY))
        y1 = min(ny - 2, math.floor(max(ay, by, cy) - OY))
        z0 = max(1, math.ceil(min(az, bz, cz) - OZ))
        z1 = min(nz - 2, math.floor(max(az, bz, cz) - OZ))
        if y0 > y1 or z0 > z1:
            continue
        e1y, e1z, e2y, e2z = by - ay, bz - az, cy - ay, cz - az
        det = e1y * e2z - e2y * e1z
        if det == 0:
            continue
        inv = 1 / det
        for k in range(z0, z1 + 1):
            pz = k + OZ - az
            for j in range(y0, y1 + 1):
                py = j + OY - ay
                w1 = (py * e2z - e2y * pz) * inv
                if w1 < 0:
                    continue
                w2 = (e1y * pz - py * e1z) * inv
                if w2 < 0 or w1 + w2 > 1:
                    continue
                cols.setdefault(j + ny * k, []).append(ax + w1 * (bx - ax) + w2 * (cx - ax))
    for c, l in cols.items():
        l.sort()
        j, k = c % ny, c // ny
        base = nx * (j + ny * k)
        for i in range(0, len(l) - 1, 2):
            a = max(1, math.ceil(l[i]))
            b = min(nx - 2, math.floor(l[i + 1]))
            if a <= b:
                vox[base + a:base + b + 1] = 1
    # surface shell
    for t in range(len(tris)):
        p = [float(v) for v in tris[t]]
        if not _finite(p):
            continue
        ax, ay, az = p[0], p[1], p[2]
        ux, uy, uz = p[3] - ax, p[4] - ay, p[5] - az
        vx, vy, vz = p[6] - ax, p[7] - ay, p[8] - az
        dx, dy, dz = ux - vx, uy - vy, uz - vz
        L = math.sqrt(max(ux * ux + uy * uy + uz * uz, vx * vx + vy * vy + vz * vz, dx * dx + dy * dy + dz * dz))
        s = max(1, min(256, math.ceil(L / 0.5)))
        for a in range(s + 1):
            fa = a / s
            for b in range(s - a + 1):
                fb = b / s
                x = _js_round(ax + ux * fa + vx * fb)
                y = _js_round(ay + uy * fa + vy * fb)
                z = _js_round(az + uz * fa + vz * fb)
                if x < 1 or y < 1 or z < 1 or x > nx - 2 or y > ny - 2 or z > nz - 2:
                    continue
                vox[x + nx * (y + ny * z)] = 1
    # flood fill fluid from the boundary
    v3 = vox.reshape(nz, ny, nx)
    seen = np.zeros((nz, ny, nx), np.uint8)
    q = deque()
    edge = np.ones((nz, ny, nx), bool)
    edge[1:-1, 1:-1, 1:-1] = False
    for z, y, x in zip(*np.nonzero(edge & (v3 == 0))):
        seen[z, y, x] = 1
        q.append((z, y, x))
    while q:
        z, y, x = q.pop()
        for dz, dy, dx in ((0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)):
            zz, yy, xx = z + dz, y + dy, x + dx
            if 0 <= zz < nz and 0 <= yy < ny and 0 <= xx < nx and not v3[zz, yy, xx] and not seen[zz, yy, xx]:
                seen[zz, yy, xx] = 1
                q.append((zz, yy, xx))
    solid = (seen.reshape(-1) == 0).astype(np.uint8)
    count = int(solid.sum())
    s3 = solid.reshape(nz, ny, nx)
    frontal = int(s3.any(axis=2).sum())
    planform = int(s3.any(axis=1).sum())
    if ground:
        s3[:, 0, :] = 2
    return solid, frontal, planform, count
