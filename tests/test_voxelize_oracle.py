"""The voxeliser oracle (oracle/voxelize_oracle.py, a restatement of web/js/voxelize.js) on
meshes whose masks are known exactly: a closed box, a box with a sealed internal pocket, a
tessellated sphere, an open triangle, non-finite and empty input."""
import numpy as np

import bodies
import voxelize_oracle as V

DIMS = (40, 24, 28)


def _box_cells(solid, dims):
    nx, ny, nz = dims
    s = solid.reshape(nz, ny, nx)
    z, y, x = np.nonzero(s == 1)
    return (x.min(), x.max(), y.min(), y.max(), z.min(), z.max()), len(x)


def test_closed_box_is_exact():
    # corners off the half-cell: parity fills x 11..20, the shell rounds the faces to 10 and 21
    solid, frontal, planform, count = V.voxelize(bodies.box_mesh((10.3, 4.4, 6.2), (20.6, 12.7, 14.1)), *DIMS, True)
    bounds, n1 = _box_cells(solid, DIMS)
    assert bounds == (10, 21, 4, 13, 6, 14)
    assert n1 == count == 12 * 10 * 9
    assert (frontal, planform) == (10 * 9, 12 * 9)
    s = solid.reshape(DIMS[2], DIMS[1], DIMS[0])
    assert (s[:, 0, :] == 2).all() and s[:, 1:, :].sum() == count  # ground layer tagged 2


def test_sealed_pocket_becomes_solid():
    outer = bodies.box_mesh((8.3, 3.4, 5.2), (30.6, 18.7, 20.1))
    inner = bodies.box_mesh((14.3, 8.4, 9.2), (22.6, 13.7, 15.1))
    a = V.voxelize(outer, *DIMS, False)
    b = V.voxelize(np.concatenate([outer, inner]), *DIMS, False)  # parity leaves the inner box empty
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]


def test_sphere_between_eroded_and_dilated_ball():
    c, r = (19.7, 11.9, 13.6), 8.0
    solid, frontal, planform, count = V.voxelize(bodies.ellipsoid_mesh(c, (r, r, r), 32, 64), *DIMS, False)
    nx, ny, nz = DIMS
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    d = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2).reshape(-1)
    assert (solid[d < r - 1.0] == 1).all()
    assert (solid[d > r + 1.0] == 0).all()
    # parity keeps the cells whose centre is inside; the shell adds ~0.7 cell over the surface,
    # i.e. about 2.1 / r of the volume (26% at r = 8)
    vol = 4 / 3 * np.pi * r ** 3
    assert 1.0 < count / vol < 1.0 + 2.6 / r


def test_open_triangle_blocks_only_its_shell():
    tri = np.array([[10.2, 5.1, 6.3, 25.7, 5.4, 7.1, 12.2, 17.8, 20.4]], np.float32)
    solid, frontal, planform, count = V.voxelize(tri, *DIMS, False)
    assert 0 < count < 600  # a one-cell-thick sheet: no enclosed volume


def test_non_finite_triangles_are_skipped_and_empty_mesh_is_fluid():
    good = bodies.box_mesh((10.3, 4.4, 6.2), (20.6, 12.7, 14.1))
    bad = np.full((2, 9), np.nan, np.float32)
    bad[1, 3] = np.inf
    a = V.voxelize(good, *DIMS, True)
    b = V.voxelize(np.concatenate([bad, good, bad]), *DIMS, True)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]
    e = V.voxelize(np.zeros((0, 9), np.float32), *DIMS, True)
    assert e[1:] == (0, 0, 0)
