"""The CUDA voxeliser (wt_voxelize through voxel.voxelize) against the oracle's restatement
of web/js/voxelize.js, bit for bit: mask, frontal and planform areas and solid count."""
import numpy as np
import pytest

import bodies
import voxelize_oracle as V

pytestmark = pytest.mark.gpu


def _rotated_ellipsoid(seed, dims):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    c = (nx * rng.uniform(0.3, 0.6), ny * rng.uniform(0.35, 0.6), nz * rng.uniform(0.35, 0.65))
    semi = (nx * rng.uniform(0.08, 0.2), ny * rng.uniform(0.1, 0.25), nz * rng.uniform(0.1, 0.25))
    t = bodies.ellipsoid_mesh(c, semi, 20, 40).reshape(-1, 3).astype(np.float64)
    a = rng.uniform(0, np.pi)
    rot = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    t = (t - c) @ rot.T + c
    return t.reshape(-1, 9).astype(np.float32)


def _soup(seed, dims, count):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    base = rng.uniform([2, 2, 2], [nx - 3, ny - 3, nz - 3], (count, 3))
    tri = np.concatenate([base, base + rng.normal(0, 3, (count, 3)), base + rng.normal(0, 3, (count, 3))], 1)
    return tri.astype(np.float32)


CASES = {
    'box': lambda d: bodies.box_mesh((10.3, 4.4, 6.2), (20.6, 12.7, 14.1)),
    'box_half_cells': lambda d: bodies.box_mesh((10.5, 4.5, 6.5), (20.5, 12.5, 14.5)),
    'pocket': lambda d: np.concatenate([bodies.box_mesh((8.3, 3.4, 5.2), (30.6, 18.7, 20.1)),
                                        bodies.box_mesh((14.3, 8.4, 9.2), (22.6, 13.7, 15.1))]),
    'ellipsoid': lambda d: _rotated_ellipsoid(3, d),
    'two_ellipsoids': lambda d: np.concatenate([_rotated_ellipsoid(4, d), _rotated_ellipsoid(5, d)]),
    'soup': lambda d: _soup(6, d, 300),
    'non_finite': lambda d: np.concatenate([np.full((3, 9), np.nan, np.float32), _rotated_ellipsoid(7, d)]),
    'empty': lambda d: np.zeros((0, 9), np.float32),
}


@pytest.mark.parametrize('name', sorted(CASES))
@pytest.mark.parametrize('dims,ground', [((40, 24, 28), True), ((64, 28, 36), False)])
def test_voxelize_matches_oracle(name, dims, ground):
    import voxel
    tris = CASES[name](dims)
    ref, frontal, planform, count = V.voxelize(tris, *dims, ground)
    got, st = voxel.voxelize(tris, dims, ground=ground)
    assert np.array_equal(got, ref), f'{name}: {int((got != ref).sum())} cells differ'
    assert (st['frontal'], st['planform'], st['count']) == (frontal, planform, count)


def test_capacity_retry_and_large_sphere():
    """More crossings than the first workspace holds (one retry), and a sphere at the
    reference's 'high' resolution: its volume and frontal area against the analytic ball."""
    import voxel
    dims = (256, 112, 136)
    c, r = (100.3, 55.6, 67.9), 50.0
    tris = np.concatenate([bodies.ellipsoid_mesh(c, (r, r, r), 64, 128)] * 5)  # 5 copies: 10 crossings per ray
    solid, st = voxel.voxelize(tris, dims, ground=True)
    assert st['crossings'] > max(4096, 4 * 112 * 136)
    vol = 4 / 3 * np.pi * r ** 3  # the shell adds ~0.7 cell over the surface: ~2.1 / r of the volume
    assert 1.0 < st['count'] / vol < 1.0 + 2.6 / r
    assert 1.0 < st['frontal'] / (np.pi * r * r) < 1.0 + 2.0 / r
    s = solid.reshape(136, 112, 256)
    assert (s[:, 0, :] == 2).all() and int((s == 1).sum()) == st['count']
