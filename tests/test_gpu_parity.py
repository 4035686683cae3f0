"""CUDA kernels (through libwt.so's C ABI, driven by the drop-in Solver) against the
golden vectors of the reference's own kernels and against the pinned oracle.

Tolerance: bit-exact. The library is built without FMA contraction and uses IEEE
division and square root, and every kernel keeps the reference's association order, so
float32 and float64 results must equal the reference's serial results exactly; fp16/bf16
storage must equal the oracle's emulation of the same rounding exactly. The fp64 force
and mass reductions sum in a different (fixed) order than the oracle, so they are
compared at a relative 1e-12.
"""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu

RANDOM_CASES = ['random_12x8x10', 'random_4x4x4', 'random_28x6x5']
# D3Q19 velocities and weights in the reference's order (server/lbm.py:15-18)
C = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, -1, 0),
     (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1), (0, 1, 1), (0, -1, -1), (0, 1, -1),
     (0, -1, 1)]
W = [1 / 3] + [1 / 18] * 6 + [1 / 36] * 12
TAGS = {'f32': ('fp32', np.float32, torch.float32), 'f64': ('fp64', np.float64, torch.float64)}


def _solver(g, precision, **kw):
    from lbm import Solver
    kw.setdefault('collision', 'exact')
    s = Solver(tuple(int(v) for v in g['dims']), 'cuda:0', precision=precision, **kw)
    s.set_solid(g['solid'])
    return s


def _load(s, which, arr):
    s.f[which].copy_(torch.from_numpy(np.ascontiguousarray(arr)).to(s.f[which].dtype))


@pytest.mark.parametrize('case', RANDOM_CASES)
@pytest.mark.parametrize('tag', ['f32', 'f64'])
def test_step_random_state_matches_reference(case, tag):
    g = golden(f'{case}_{tag}.npz')
    prec, nd, td = TAGS[tag]
    s = _solver(g, prec)
    _load(s, 0, g['f0_in'])
    _load(s, 1, g['f1_in'])
    s.mac[0].copy_(torch.from_numpy(g['mac_in']))
    torch.cuda.synchronize()  # the copies ran on torch's stream, the kernels run on the Solver's
    p = dict(uIn=float(g['uin']), tau=float(g['tau']), smag=float(g['smag']))
    done = 0
    for k in g['steps']:
        s.step(int(k) - done, p)
        done = int(k)
        s.synchronize()
        f_cur = s.f[s.cur].cpu().numpy()
        f_old = s.f[1 - s.cur].cpu().numpy()
        mac = s.mac[s.cur].cpu().numpy()
        assert np.array_equal(f_cur, g[f'f_cur_{k}']), f'f after {k} steps: max diff {np.abs(f_cur - g[f"f_cur_{k}"]).max()}'
        assert np.array_equal(f_old, g[f'f_old_{k}'])
        assert np.array_equal(mac, g[f'mac_{k}'])
        f6 = s.forces6()
        np.testing.assert_allclose(f6[:3], g[f'forces_{k}'].astype(np.float64), rtol=2e-5, atol=1e-6)


@pytest.mark.parametrize('tag', ['f32', 'f64'])
def test_sphere_100_steps_matches_reference(tag, oracle_mod):
    g = golden(f'sphere_32x16x16_{tag}.npz')
    prec, nd, td = TAGS[tag]
    s = _solver(g, prec)
    p = dict(uIn=float(g['uin']), tau=float(g['tau']), smag=float(g['smag']))
    s.reset(p['uIn'])
    s.step(50, p)
    s.synchronize()
    assert np.array_equal(s.f[s.cur].cpu().numpy(), g['f_cur_50'])
    s.step(50, p)
    s.synchronize()
    assert np.array_equal(s.f[s.cur].cpu().numpy(), g['f_cur'])
    assert np.array_equal(s.f[1 - s.cur].cpu().numpy(), g['f_old'])
    assert np.array_equal(s.mac[s.cur].cpu().numpy(), g['mac'])
    # forces: the reference's float sum (tid order) to float rounding; the oracle's fp64 sum
    # of the same per-cell values to 1e-12
    L = oracle_mod.Lattice(tuple(int(v) for v in g['dims']), oracle_mod.F32 if tag == 'f32' else oracle_mod.F64)
    L.solid[:] = g['solid']
    L.f[0][:] = g['f_cur']
    _, d64, b64 = L.forces()
    f6 = s.forces6()
    np.testing.assert_allclose(f6[:3], d64, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(f6[3:], b64, rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(f6[:3], g['forces'].astype(np.float64), rtol=2e-5, atol=1e-7)
    np.testing.assert_allclose(s.mass(), L.mass(), rtol=1e-13)


def test_frame_kernels_match_reference():
    g = golden('sphere_32x16x16_f32.npz')
    s = _solver(g, 'fp32')
    dims = tuple(int(v) for v in g['dims'])
    s.mac[s.cur].copy_(torch.from_numpy(g['mac']))
    dt, uin, max_age, seed, sx, scy, scz, shy, shz = (float(v) for v in g['adv_params'])
    # particles: place the golden inputs, advect once with the golden seed
    s.num_p = len(g['adv_pos_in'])
    s.pos = torch.from_numpy(g['adv_pos_in'].copy()).cuda()
    s.spd = torch.ones(s.num_p, dtype=torch.float32, device='cuda')
    s.q16 = torch.zeros(s.num_p * 4, dtype=torch.int16, device='cuda')
    s.q8 = torch.zeros(s.num_p, dtype=torch.uint8, device='cuda')
    torch.cuda.synchronize()
    s.seed = int(seed) - 1
    p = dict(uIn=uin, tau=0.506, smag=0.16, maxAge=max_age, seedX=sx, seedCy=scy, seedCz=scz, seedHy=shy,
             seedHz=shz, lref=8.0)
    s.seed += 1
    s._advect(dt, p)
    s.synchronize()
    assert np.array_equal(s.pos.cpu().numpy(), g['adv_pos'])
    assert np.array_equal(s.spd.cpu().numpy(), g['adv_spd'])
    s.set_surface(g['cp_verts'], g['cp_norms'])
    for axis in (0, 1, 2):
        for field in range(4):
            a = g[f'slice_{axis}_{field}_args']
            p['slice'] = dict(axis=int(a[0]), index=int(a[1]), field=int(a[2]), vmin=float(a[4]), vmax=float(a[5]))
            p['lref'] = float(a[3])
            out = s.frame(p, want_cp=True)
            assert np.array_equal(out['slice'], g[f'slice_{axis}_{field}']), (axis, field)
            assert (out['sliceW'], out['sliceH'], out['sliceAxis']) == s.slice_dims(axis) + (axis,)
    assert np.array_equal(out['parts16'], g['pack_q16'])
    assert np.array_equal(out['parts8'], g['pack_q8'])
    assert np.array_equal(out['cp'], g['cp'])
    assert len(out['forces']) == 3


def test_frame_kernels_at_the_edges():
    """Slices of the first and last plane of every axis (and indices outside, which the Solver
    clamps as server/lbm.py:467 does), particles packed and advected at and beyond the domain
    edges, and surface points at the corners and outside, against the oracle."""
    import oracle
    dims = (20, 9, 7)
    nx, ny, nz = dims
    n = nx * ny * nz
    rng = np.random.default_rng(31)
    solid = _random_case(dims, 31)
    mac = np.empty((n, 4), np.float32)
    mac[:, :3] = rng.uniform(-0.12, 0.12, (n, 3))
    mac[:, 3] = rng.uniform(0.9, 1.1, n)
    s = _solver(dict(dims=np.array(dims), solid=solid), 'fp32')
    s.mac[s.cur].copy_(torch.from_numpy(mac))
    torch.cuda.synchronize()
    uin = 0.06
    p = dict(uIn=uin, tau=0.51, smag=0.16, lref=6.0, maxAge=50.0, seedX=2.0, seedCy=4.0, seedCz=3.0, seedHy=2.5,
             seedHz=2.0)
    for axis in range(3):
        dim = dims[axis]
        for index in (0, dim - 1, -4, dim + 5):
            for field in range(4):
                p['slice'] = dict(axis=axis, index=index, field=field, vmin=0.0, vmax=1.4)
                out = s.frame(p, want_cp=False)
                ref = oracle.slice_(mac, solid, dims, axis, max(0, min(dim - 1, index)), field, uin, p['lref'], 0.0,
                                    1.4)
                assert np.array_equal(out['slice'], ref), (axis, index, field)
    p['slice'] = None
    # particles on the faces, corners and outside; speeds at and beyond the packing range
    xs = [0.0, nx - 1.0, -3.0, nx + 2.5, 0.5, nx - 3.0, 1e6, -1e6]
    ys = [0.0, ny - 1.0, ny + 4.0, -2.0, 0.5, ny - 1.5]
    zs = [0.0, nz - 1.0, -1.0, nz + 3.0, 0.5, nz - 1.5]
    pos = np.array([(x, y, z, a) for x in xs for y in ys for z in zs for a in (0.0, 3.0)], np.float32)
    spd = np.resize(np.array([0.0, 1.99, 2.0, 5.0, -1.0, 0.004], np.float32), len(pos))
    s.num_p = len(pos)
    s.pos = torch.from_numpy(pos.copy()).cuda()
    s.spd = torch.from_numpy(spd.copy()).cuda()
    s.q16 = torch.zeros(s.num_p * 4, dtype=torch.int16, device='cuda')
    s.q8 = torch.zeros(s.num_p, dtype=torch.uint8, device='cuda')
    torch.cuda.synchronize()
    out = s.frame(p, want_cp=False)
    q16, q8 = oracle.pack(pos, spd, dims)
    assert np.array_equal(out['parts16'].view(np.uint16), q16)
    assert np.array_equal(out['parts8'], q8)
    s.seed = 40
    s._advect(3.0, p)
    s.synchronize()
    pos_o, spd_o = pos.copy(), spd.copy()
    oracle.advect(pos_o, spd_o, mac, solid, dims, 3.0, uin, p['maxAge'], 40, p['seedX'], p['seedCy'], p['seedCz'],
                  p['seedHy'], p['seedHz'])
    assert np.array_equal(s.pos.cpu().numpy(), pos_o)
    assert np.array_equal(s.spd.cpu().numpy(), spd_o)
    # surface points at the corners, on the faces and outside, normals along each axis and diagonals
    verts = np.array([(x, y, z) for x in (0.0, nx - 1.0, -2.0, nx + 1.0, 3.3) for y in (0.0, ny - 1.0, 4.6)
                      for z in (0.0, nz - 1.0, -1.5, 2.2)], np.float32)
    dirs = np.array([(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (0.6, 0.8, 0),
                     (0, -0.6, 0.8)], np.float32)
    norms = np.resize(dirs, (len(verts), 3)).astype(np.float32)
    s.set_surface(verts, norms)
    out = s.frame(p, want_cp=True)
    assert np.array_equal(out['cp'], oracle.cp(mac, solid, verts, norms, dims, uin))


def _random_case(dims, seed, belt=True):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    n = nx * ny * nz
    r = rng.random(n)
    solid = np.zeros(n, np.uint8)
    solid[r < 0.08] = 1
    solid[(r > 0.5) & (r < 0.52)] = 2
    if belt:
        solid.reshape(nz, ny, nx)[:, 0, :] = 2
    return solid


@pytest.mark.parametrize('prec_name,oprec,shift', [('fp32', 0, 'free-stream'), ('fp16', 1, 'free-stream'),
                                                    ('bf16', 2, 'free-stream'), ('fp16', 1, 'rest'),
                                                    ('bf16', 2, 'rest'), ('fp64', 3, 'free-stream')])
@pytest.mark.parametrize('dims', [(64, 24, 20), (34, 9, 7)])
def test_random_obstacles_match_oracle(oracle_mod, prec_name, oprec, shift, dims):
    """Larger grids than the goldens, every storage precision (half-width storage shifted by
    the free-stream equilibrium and by the rest weights), against the pinned oracle."""
    solid = _random_case(dims, 5)
    uin, tau, smag = 0.06, 0.52, 0.16
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name, shift=shift)
    s.reset(uin)
    if oprec in (1, 2):
        assert float(s.grid.shift_u) == (float(np.float32(uin)) if shift == 'free-stream' else 0.0)
    L = oracle_mod.Lattice(dims, oprec, shift_u=float(s.grid.shift_u))
    L.solid[:] = solid
    L.reset(uin)
    p = dict(uIn=uin, tau=tau, smag=smag)
    for chunk in (1, 4, 7):
        s.step(chunk, p)
        L.step(chunk, uin, tau, smag)
        s.synchronize()
        dev = s.f[s.cur].cpu()
        if oprec == 2:
            dev = dev.view(torch.int16).numpy().view(np.uint16)
        else:
            dev = dev.numpy()
        assert np.array_equal(dev, L.f[L.cur]), f'{prec_name} after chunk {chunk}'
        assert np.array_equal(s.mac[s.cur].cpu().numpy(), L.mac)
    _, d64, b64 = L.forces()
    f6 = s.forces6()
    np.testing.assert_allclose(f6[:3], d64, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(f6[3:], b64, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(s.mass(), L.mass(), rtol=1e-13)


def test_config1_sphere_2000_steps_matches_oracle(oracle_mod):
    """The reference's CPU-runnable workload at its full size: 128x64x64, sphere r = 8 at
    (40, 32, 32), no-slip floor, u = 0.05, nu = 0.002, 2000 steps from equilibrium. Populations
    and mac bit for bit every 50 steps; the drag and lift (fp64 sums of all links, and without
    the floor's) and Cd/Cl on the sphere's frontal area against the oracle's at every check."""
    import os
    import bodies
    dims, solid, p = bodies.config1()
    oracle_mod.set_threads(os.cpu_count() or 1)
    s = _solver(dict(dims=np.array(dims), solid=solid), 'fp32')
    s.reset(p['uIn'])
    L = oracle_mod.Lattice(dims, 0)
    L.solid[:] = solid
    L.reset(p['uIn'])
    frontal = bodies.areas(solid, dims)[0]
    q = 0.5 * p['uIn'] ** 2 * frontal
    for k in range(40):
        s.step(50, p)
        L.step(50, p['uIn'], p['tau'], p['smag'])
        s.synchronize()
        assert np.array_equal(s.f[s.cur].cpu().numpy(), L.f[L.cur]), f'populations after {50 * (k + 1)} steps'
        assert np.array_equal(s.mac[s.cur].cpu().numpy(), L.mac), f'mac after {50 * (k + 1)} steps'
        _, d64, b64 = L.forces()
        f6 = s.forces6()
        np.testing.assert_allclose(f6[:3], d64, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose(f6[3:], b64, rtol=1e-12, atol=1e-14)
        np.testing.assert_allclose([f6[3] / q, f6[4] / q], [b64[0] / q, b64[1] / q], rtol=1e-12, atol=1e-14)


@pytest.mark.parametrize('prec_name,oprec', [('fp32', 0), ('fp16', 1)])
def test_benchmark_workload_full_size_matches_oracle(oracle_mod, prec_name, oprec):
    """The 512x256x256 benchmark body (33.5M cells, the largest configuration) for 6 steps, the
    last writing mac for every cell: populations, mac, forces and mass against the oracle."""
    import os
    import bodies
    dims, solid, p = bodies.config2()
    oracle_mod.set_threads(os.cpu_count() or 1)
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name)
    s.reset(p['uIn'])
    L = oracle_mod.Lattice(dims, oprec, shift_u=float(s.grid.shift_u))
    L.solid[:] = solid
    L.reset(p['uIn'])
    s.step(6, p)
    L.step(6, p['uIn'], p['tau'], p['smag'])
    s.synchronize()
    assert np.array_equal(s.f[s.cur].cpu().numpy(), L.f[L.cur])
    assert np.array_equal(s.mac[s.cur].cpu().numpy(), L.mac)
    _, d64, b64 = L.forces()
    f6 = s.forces6()
    np.testing.assert_allclose(f6[:3], d64, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(f6[3:], b64, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(s.mass(), L.mass(), rtol=1e-13)


def _degenerate(name):
    """Grids at and near the smallest the library accepts, and masks with nothing to do."""
    if name == 'min_4x3x3_fluid':
        return (4, 3, 3), np.zeros(36, np.uint8)
    if name == 'min_4x3x3_belt':
        s = np.zeros(36, np.uint8)
        s.reshape(3, 3, 4)[:, 0, :] = 2
        return (4, 3, 3), s
    if name == 'row_34x3x3':  # one interior row
        return (34, 3, 3), _random_case((34, 3, 3), 21)
    if name == 'short_4x10x7':  # the inlet and outlet columns are neighbours of one interior pair
        return (4, 10, 7), _random_case((4, 10, 7), 22)
    if name == 'thin_6x3x5':
        return (6, 3, 5), _random_case((6, 3, 5), 23)
    if name == 'all_solid_10x5x5':
        return (10, 5, 5), np.ones(250, np.uint8)
    if name == 'one_fluid_cell_8x5x5':
        s = np.ones(200, np.uint8)
        s[3 + 8 * (2 + 5 * 2)] = 0
        return (8, 5, 5), s
    raise KeyError(name)


DEGENERATE = ['min_4x3x3_fluid', 'min_4x3x3_belt', 'row_34x3x3', 'short_4x10x7', 'thin_6x3x5', 'all_solid_10x5x5',
              'one_fluid_cell_8x5x5']


@pytest.mark.parametrize('prec_name,oprec', [('fp32', 0), ('fp16', 1), ('fp64', 3)])
@pytest.mark.parametrize('case', DEGENERATE)
def test_degenerate_grids_match_oracle(oracle_mod, case, prec_name, oprec):
    """Smallest and thinnest grids (every cell a face or next to one), an all-solid mask and a
    single fluid cell, in every admissible tile, bit for bit against the oracle."""
    import autotune
    dims, solid = _degenerate(case)
    uin, tau, smag = 0.07, 0.52, 0.16
    p = dict(uIn=uin, tau=tau, smag=smag)
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name)
    L = oracle_mod.Lattice(dims, oprec, shift_u=float(np.float32(uin)) if oprec in (1, 2) else 0.0)
    L.solid[:] = solid
    L.reset(uin)
    L.step(6, uin, tau, smag)
    tiles = [t[0] for t in autotune.admissible(s)]
    assert tiles
    for tile in tiles:
        s.set_tile(tile)
        s.reset(uin)
        s.cur = 0
        for chunk in (1, 2, 3):
            s.step(chunk, p)
        s.synchronize()
        assert np.array_equal(s.f[s.cur].cpu().numpy(), L.f[L.cur]), f'{case} tile {tile}'
        assert np.array_equal(s.mac[s.cur].cpu().numpy(), L.mac), f'{case} tile {tile}'
    _, d64, b64 = L.forces()
    f6 = s.forces6()
    np.testing.assert_allclose(f6[:3], d64, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(s.mass(), L.mass(), rtol=1e-13)


def test_link_list_matches_mask():
    dims = (48, 20, 18)
    solid = _random_case(dims, 9)
    s = _solver(dict(dims=np.array(dims), solid=solid), 'fp32')
    nx, ny, nz = dims
    from bodies import C
    expect_cells, expect_masks = [], []
    v = solid.reshape(nz, ny, nx)
    for z in range(1, nz - 1):
        for y in range(1, ny - 1):
            for x in range(1, nx - 1):
                if v[z, y, x]:
                    continue
                m = 0
                for i in range(1, 19):
                    if v[z + C[i][2], y + C[i][1], x + C[i][0]] == 1:
                        m |= 1 << (i - 1)
                if m:
                    expect_cells.append(x + nx * (y + ny * z))
                    expect_masks.append(m)
    assert s.n_links == len(expect_cells)
    assert np.array_equal(s.link_cells[:s.n_links].cpu().numpy(), np.array(expect_cells, np.int32))
    assert np.array_equal(s.link_masks[:s.n_links].cpu().numpy().view(np.uint32), np.array(expect_masks, np.uint32))


def test_repeatable_bitwise():
    dims = (64, 24, 20)
    solid = _random_case(dims, 3)
    outs = []
    for _ in range(2):
        s = _solver(dict(dims=np.array(dims), solid=solid), 'fp32')
        s.reset(0.05)
        s.step(20, dict(uIn=0.05, tau=0.51, smag=0.16))
        outs.append((s.populations(), s.forces6(), s.mass()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
    assert outs[0][2] == outs[1][2]


@pytest.mark.parametrize('prec_name,oprec', [('fp32', 0), ('fp16', 1), ('bf16', 2), ('fp64', 3)])
def test_every_tile_variant_matches_oracle(oracle_mod, prec_name, oprec):
    """All tile shapes of the step kernel compute the same bits."""
    import autotune
    dims = (64, 20, 12)
    solid = _random_case(dims, 17)
    uin, tau, smag = 0.05, 0.51, 0.16
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name)
    s.reset(uin)
    L = oracle_mod.Lattice(dims, oprec, shift_u=float(s.grid.shift_u))
    L.solid[:] = solid
    L.reset(uin)
    L.step(5, uin, tau, smag)
    tiles = autotune.admissible(s)
    assert len(tiles) >= 4
    for tile in tiles:
        s.set_tile(tile[0])
        s.reset(uin)
        s.cur = 0
        s.step(5, dict(uIn=uin, tau=tau, smag=smag))
        s.synchronize()
        dev = s.f[s.cur].cpu()
        dev = dev.view(torch.int16).numpy().view(np.uint16) if oprec == 2 else dev.numpy()
        assert np.array_equal(dev, L.f[L.cur]), f'tile {tile}'
        assert np.array_equal(s.mac[s.cur].cpu().numpy(), L.mac), f'tile {tile}'


def test_autotune_picks_a_tile():
    import autotune
    dims = (64, 24, 20)
    s = _solver(dict(dims=np.array(dims), solid=_random_case(dims, 2)), 'fp32')
    s.reset(0.05)
    tile, ms = autotune.tune(s, dict(uIn=0.05, tau=0.51, smag=0.16), steps=2, warm=1, repeats=1, force=True)
    assert tile in ms and s.tile == tile and all(v > 0 for v in ms.values())


# The fast form takes reciprocals and square roots from the special-function unit (about
# 1 float ulp), the oracle restates the same algebra with IEEE operations; after 5 steps
# the populations must agree to these absolute tolerances (f is O(0.03..0.33)):
FAST_ATOL = {'fp32': 2e-6, 'fp16': 3e-5, 'bf16': 3e-4, 'fp64': 1e-12}


@pytest.mark.parametrize('prec_name,oprec', [('fp32', 0), ('fp16', 1), ('bf16', 2), ('fp64', 3)])
@pytest.mark.parametrize('dims', [(64, 24, 20), (34, 9, 7)])
def test_fast_collision_matches_oracle(oracle_mod, prec_name, oprec, dims):
    """The moment-space collision in every storage precision and tile against the oracle's
    restatement of the same operation sequence."""
    import autotune
    solid = _random_case(dims, 23)
    uin, tau, smag = 0.07, 0.515, 0.16
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name, collision='fast')
    s.reset(uin)
    L = oracle_mod.Lattice(dims, oprec, collision=1, shift_u=float(s.grid.shift_u))
    L.solid[:] = solid
    L.reset(uin)
    L.step(5, uin, tau, smag)
    ref = L.populations()
    p = dict(uIn=uin, tau=tau, smag=smag)
    tiles = autotune.admissible(s)
    assert tiles
    for tile in tiles:
        s.set_tile(tile[0])
        s.reset(uin)
        s.cur = 0
        s.step(5, p)
        got = s.populations()
        err = np.abs(got - ref).max()
        assert err <= FAST_ATOL[prec_name], f'{prec_name} tile {tile}: max |df| {err}'
        np.testing.assert_allclose(s.macro(), L.mac.astype(np.float64), atol=20 * FAST_ATOL[prec_name], rtol=0)


def _random_flow(s, seed, umax=0.3):
    """Equilibrium populations at random rho in [0.95, 1.05] and velocities uniform in
    [-umax, umax]^3 (|u| up to 0.52: some cells hit the 0.35 clamp, their neighbours not)."""
    rng = np.random.default_rng(seed)
    c = np.array(C, np.float64)
    w = np.array(W, np.float64)
    u = rng.uniform(-umax, umax, (s.n, 3))
    rho = rng.uniform(0.95, 1.05, s.n)
    cu = u @ c.T
    f = (w[None, :] * rho[:, None] * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * (u * u).sum(1)[:, None])).T
    if s.precision in (1, 2):  # shifted storage holds f - e
        from lbm import shift_values
        f = f - shift_values(float(s.grid.shift_u)).astype(np.float64)[:, None]
    _load(s, s.cur, f.reshape(-1))


@pytest.mark.parametrize('prec_name', ['fp32', 'fp16', 'bf16'])
@pytest.mark.parametrize('dims', [(64, 24, 20), (48, 9, 7)])
def test_fast_pair_collision_same_bits_in_every_tile(prec_name, dims):
    """Tiles with two or four cells per thread run the fast collision on cell pairs with
    sm_100's paired fp32 instructions, which round each lane like the one-lane forms: every
    tile must give the bits of the one-cell tile, including cells whose pair partner is
    clamped, in the outlet sponge or next to a wall."""
    import autotune
    solid = _random_case(dims, 29)
    p = dict(uIn=0.07, tau=0.512, smag=0.16)
    s = _solver(dict(dims=np.array(dims), solid=solid), prec_name, collision='fast')
    tiles = [t[0] for t in autotune.admissible(s)]
    assert 1 in tiles and any(t[1] >= 2 for t in autotune.admissible(s))
    out = {}
    for tile in [1] + [t for t in tiles if t != 1]:
        s.set_tile(tile)
        s.reset(p['uIn'])
        s.cur = 0
        _random_flow(s, 5)
        s.step(3, p)
        out[tile] = (s.populations(), s.macro())
        assert np.array_equal(out[tile][0], out[1][0]), f'{prec_name} tile {tile}: populations'
        assert np.array_equal(out[tile][1], out[1][1]), f'{prec_name} tile {tile}: mac'


def test_fast_collision_close_to_exact():
    """Both collision forms evaluate the same physics: after 100 steps of flow past an
    obstacle the fp32 populations agree to 1e-5 relative (the tolerance the reference
    comparison allows)."""
    import bodies
    dims = (64, 32, 32)
    solid = bodies.sphere_tunnel(dims, (20, 16, 16), 5.0, floor='belt')
    p = dict(uIn=0.05, tau=0.506, smag=0.16)
    out = []
    for form in ('exact', 'fast'):
        s = _solver(dict(dims=np.array(dims), solid=solid), 'fp32', collision=form)
        s.reset(p['uIn'])
        s.step(100, p)
        out.append(s.populations())
    rel = np.abs(out[1] - out[0]) / np.abs(out[0])
    assert rel.max() < 1e-5, rel.max()
