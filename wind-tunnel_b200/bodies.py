"""Seeded synthetic obstacles, standing in for the masks the reference's browser client
voxelises from STL uploads (web/js/voxelize.js) and the surface mesh it uploads.

Mask semantics are the reference's: 0 fluid, 1 solid, 2 moving ground belt on the y = 0
plane (voxelize.js:112). Solid cells are kept off the domain faces (x, z in [1, n-2]),
as the client's voxeliser does (voxelize.js:47, 67). Frontal and planform areas follow
voxelize.js:99-110 (projections counted before the belt is added).
"""
import numpy as np

Q = 19
C = np.array([(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
              (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
              (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)])


def _grid(dims):
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nx, dtype=np.float32), indexing='ij', sparse=True)
    return x, y, z


def sphere(dims, centre, radius):
    """Cell-centre-inside sphere: solid = 1 where (x-cx)^2 + (y-cy)^2 + (z-cz)^2 <= r^2."""
    x, y, z = _grid(dims)
    inside = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2 <= radius * radius
    return inside.astype(np.uint8).reshape(-1)


def ellipsoid_union(dims, count, seed, semi=(10.0, 60.0), scale=1.0, floor='belt'):
    """Union of `count` axis-aligned ellipsoids resting on the floor (centre y = 1 + b),
    semi-axes uniform in `semi` cells times `scale`, centres drawn from PCG64(seed)."""
    nx, ny, nz = dims
    rng = np.random.Generator(np.random.PCG64(seed))
    x, y, z = _grid(dims)
    solid = np.zeros((nz, ny, nx), np.uint8)
    params = []
    for _ in range(count):
        a, b, c = (rng.uniform(semi[0], semi[1], 3) * scale).tolist()
        b = min(b, 0.45 * ny)
        a = min(a, 0.2 * nx)
        c = min(c, 0.3 * nz)
        cx = rng.uniform(0.25 * nx, 0.5 * nx)
        cz = rng.uniform(0.5 * nz - 0.15 * nz, 0.5 * nz + 0.15 * nz)
        cy = 1.0 + b
        params.append((cx, cy, cz, a, b, c))
        for zs in range(0, nz, 64):  # slab-wise to bound temporaries at 33.5M cells
            zz = z[zs:zs + 64]
            inside = ((x - cx) / a) ** 2 + ((y - cy) / b) ** 2 + ((zz - cz) / c) ** 2 <= 1.0
            solid[zs:zs + 64] |= inside.astype(np.uint8)
    solid = _finish(solid.reshape(-1), floor, dims)
    return solid, params


def _finish(solid, floor, dims=None):
    s = solid.reshape(-1).copy()
    if dims is not None:
        nx, ny, nz = dims
        v = s.reshape(nz, ny, nx)
        v[:, :, 0] = 0
        v[:, :, nx - 1] = 0
        v[0] = 0
        v[nz - 1] = 0
        v[:, ny - 1] = 0
    return s if floor is None else _floor(s, floor, dims)


def _floor(s, floor, dims):
    if dims is None:
        raise ValueError('floor needs dims')
    nx, ny, nz = dims
    v = s.reshape(nz, ny, nx)
    v[:, 0, :] = {'noslip': 1, 'belt': 2}[floor]
    return s


def sphere_tunnel(dims, centre, radius, floor=None):
    """Sphere plus an optional floor: 'noslip' (y = 0 plane set to 1) or 'belt' (set to 2)."""
    s = sphere(dims, centre, radius)
    return s if floor is None else _floor(s, floor, dims)


def areas(solid, dims):
    """(frontal, planform) in cells^2: y-z and x-z projections of solid == 1 cells,
    excluding the y = 0 plane (voxelize.js:99-110 counts before the belt is set)."""
    nx, ny, nz = dims
    v = solid.reshape(nz, ny, nx) == 1
    v = v.copy()
    v[:, 0, :] = False
    frontal = int(v.any(axis=2).sum())
    planform = int(v.any(axis=1).sum())
    return frontal, planform


def surface_points(solid, dims, max_points=None):
    """Boundary points for surface pressure: every interior fluid cell with a solid == 1
    neighbour along the 18 links, excluding links into the y = 0 plane. The normal is the
    normalised sum of -c_i over those links (the mask gradient); the point sits half a
    cell from the cell centre towards the wall. Returns (verts, norms), float32 (V, 3)."""
    nx, ny, nz = dims
    v = (solid.reshape(nz, ny, nx) == 1)
    v[:, 0, :] = False
    fluid = solid.reshape(nz, ny, nx) == 0
    acc = np.zeros((nz, ny, nx, 3), np.float32)
    hit = np.zeros((nz, ny, nx), bool)
    for i in range(1, Q):
        cx, cy, cz = C[i]
        sh = np.zeros_like(v)
        # sh[z, y, x] = v[z + cz, y + cy, x + cx]
        zs = slice(max(0, -cz), nz - max(0, cz))
        ys = slice(max(0, -cy), ny - max(0, cy))
        xs = slice(max(0, -cx), nx - max(0, cx))
        zd = slice(max(0, cz), nz - max(0, -cz))
        yd = slice(max(0, cy), ny - max(0, -cy))
        xd = slice(max(0, cx), nx - max(0, -cx))
        sh[zs, ys, xs] = v[zd, yd, xd]
        hit |= sh
        acc[sh] -= C[i].astype(np.float32)
    inner = np.zeros_like(hit)
    inner[1:-1, 1:-1, 1:-1] = True
    sel = hit & fluid & inner
    zi, yi, xi = np.nonzero(sel)
    nrm = acc[zi, yi, xi]
    ln = np.linalg.norm(nrm, axis=1, keepdims=True)
    ok = ln[:, 0] > 0
    nrm = nrm[ok] / ln[ok]
    pts = np.stack([xi[ok], yi[ok], zi[ok]], axis=1).astype(np.float32) - 0.5 * nrm
    if max_points is not None and len(pts) > max_points:
        keep = np.linspace(0, len(pts) - 1, max_points).astype(np.int64)
        pts, nrm = pts[keep], nrm[keep]
    return np.ascontiguousarray(pts, np.float32), np.ascontiguousarray(nrm, np.float32)


# ---- the workloads of the benchmark configurations ----

def config1():
    """128x64x64, sphere r = 8 at (40, 32, 32), no-slip floor (y = 0 set to 1);
    u = 0.05, nu = 0.002 (tau = 0.506), Cs = 0.16."""
    dims = (128, 64, 64)
    solid = sphere_tunnel(dims, (40, 32, 32), 8.0, floor='noslip')
    return dims, solid, dict(uIn=0.05, tau=3 * 0.002 + 0.5, smag=0.16)


def config2(scale=1.0, seed=2024):
    """512x256x256 (scaled), union of 6 seeded ellipsoids (semi-axes 10-60 cells) resting on
    a moving belt; u = 0.05, nu = 0.001 (tau = 0.503), Cs = 0.16."""
    dims = (int(512 * scale), int(256 * scale), int(256 * scale))
    solid, _ = ellipsoid_union(dims, 6, seed, scale=scale, floor='belt')
    return dims, solid, dict(uIn=0.05, tau=3 * 0.001 + 0.5, smag=0.16)


def config4(count=24, seed=4, cells=(0.5e6, 8e6)):
    """Batching workload: `count` tunnels, cell counts log-uniform in `cells`, aspect 2:1:1
    (nx = 2 ny = 2 nz, nx a multiple of 16), each with its own seeded union of 1-6 ellipsoids
    on a moving belt, u0 uniform in [0.03, 0.08], nu uniform in [0.001, 0.01] (tau = 3 nu + 1/2).
    Returns [(dims, solid, params)]."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for t in range(count):
        n = float(np.exp(rng.uniform(np.log(cells[0]), np.log(cells[1]))))
        nx = max(32, int(round((4.0 * n) ** (1.0 / 3.0) / 16.0)) * 16)
        dims = (nx, nx // 2, nx // 2)
        k = int(rng.integers(1, 7))
        solid, _ = ellipsoid_union(dims, k, int(rng.integers(1 << 31)), scale=nx / 512.0, floor='belt')
        u0 = float(rng.uniform(0.03, 0.08))
        nu = float(rng.uniform(0.001, 0.01))
        out.append((dims, solid, dict(uIn=u0, tau=3.0 * nu + 0.5, smag=0.16)))
    return out


# ---- triangle meshes (lattice coordinates) for the voxeliser ----
def box_mesh(lo, hi):
    """Closed axis-aligned box [lo, hi] as 12 triangles, float32 (12, 9)."""
    (x0, y0, z0), (x1, y1, z1) = lo, hi
    v = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0],
                  [x0, y0, z1], [x1, y0, z1], [x1, y1, z1], [x0, y1, z1]], np.float64)
    quads = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    tris = []
    for a, b, c, d in quads:
        tris += [v[[a, b, c]].reshape(-1), v[[a, c, d]].reshape(-1)]
    return np.array(tris, np.float32)


def ellipsoid_mesh(centre, semi, n_lat=24, n_lon=48):
    """Closed UV-tessellated ellipsoid, float32 (T, 9): rings of latitude between the poles."""
    cx, cy, cz = centre
    a, b, c = semi
    th = np.linspace(0.0, np.pi, n_lat + 1)
    ph = np.linspace(0.0, 2.0 * np.pi, n_lon + 1)

    def pt(i, j):
        return (cx + a * np.sin(th[i]) * np.cos(ph[j]), cy + b * np.cos(th[i]), cz + c * np.sin(th[i]) * np.sin(ph[j]))

    tris = []
    for i in range(n_lat):
        for j in range(n_lon):
            p00, p01, p10, p11 = pt(i, j), pt(i, j + 1), pt(i + 1, j), pt(i + 1, j + 1)
            if i > 0:
                tris.append(p00 + p10 + p01)
            if i < n_lat - 1:
                tris.append(p01 + p10 + p11)
    return np.array(tris, np.float32)

