"""Pin the C++ oracle to golden vectors made from the reference's own kernel code.

The fixtures under tests/golden/ were produced by tests/golden/make_golden.py, which
runs server/lbm.py of RICKxxROLLING/wind-tunnel (generated init/step/force kernels and
the hand-written particle/slice/cp kernels) serially under a stub warp module. The
oracle must reproduce them bit for bit in float32 and float64; only then is it trusted
as the parity checker for the CUDA kernels.
"""
import numpy as np
import pytest

from conftest import golden

RANDOM_CASES = ['random_12x8x10', 'random_4x4x4', 'random_28x6x5']


def _lattice_from(oracle_mod, g, prec, dtype):
    L = oracle_mod.Lattice(tuple(int(v) for v in g['dims']), prec)
    L.solid[:] = g['solid']
    return L


@pytest.mark.parametrize('case', RANDOM_CASES)
@pytest.mark.parametrize('tag,prec', [('f32', 0), ('f64', 3)])
@pytest.mark.parametrize('serial', [True, False])
def test_step_random_state_bit_exact(oracle_mod, case, tag, prec, serial):
    """Far-from-equilibrium states: velocity clamp, rho clamp at faces, outlet ux < 0,
    bounce-back, belt and mask value 3 all fire; serial and parallel orders agree."""
    g = golden(f'{case}_{tag}.npz')
    L = _lattice_from(oracle_mod, g, prec, None)
    L.f[0][:] = g['f0_in']
    L.f[1][:] = g['f1_in']
    L.mac[:] = g['mac_in']
    done = 0
    for k in g['steps']:
        L.step(int(k) - done, g['uin'], g['tau'], g['smag'], serial=serial)
        done = int(k)
        assert np.array_equal(L.f[L.cur], g[f'f_cur_{k}']), f'f after {k} steps'
        assert np.array_equal(L.f[1 - L.cur], g[f'f_old_{k}']), f'old f after {k} steps'
        assert np.array_equal(L.mac, g[f'mac_{k}']), f'mac after {k} steps'
        ref, _, _ = L.forces()
        assert np.array_equal(ref, g[f'forces_{k}']), f'forces after {k} steps'


@pytest.mark.parametrize('tag,prec', [('f32', 0), ('f64', 3)])
def test_sphere_100_steps_bit_exact(oracle_mod, tag, prec):
    """Inlet flow past a sphere over a moving belt, 100 steps from the reference's reset."""
    g = golden(f'sphere_32x16x16_{tag}.npz')
    L = _lattice_from(oracle_mod, g, prec, None)
    L.reset(g['uin'])
    assert np.array_equal(L.f[0], g['init_f'])
    assert np.array_equal(L.mac, g['init_mac'])
    L.step(50, g['uin'], g['tau'], g['smag'])
    assert np.array_equal(L.f[L.cur], g['f_cur_50'])
    L.step(50, g['uin'], g['tau'], g['smag'])
    assert np.array_equal(L.f[L.cur], g['f_cur'])
    assert np.array_equal(L.f[1 - L.cur], g['f_old'])
    assert np.array_equal(L.mac, g['mac'])
    ref, d64, _ = L.forces()
    assert np.array_equal(ref, g['forces'])
    # the fp64 accumulation of the same per-cell sums agrees to float rounding
    np.testing.assert_allclose(d64, g['forces'].astype(np.float64), rtol=1e-5, atol=1e-7)


def test_frame_kernels_bit_exact(oracle_mod):
    g = golden('sphere_32x16x16_f32.npz')
    dims = tuple(int(v) for v in g['dims'])
    mac = np.ascontiguousarray(g['mac'])
    solid = g['solid']
    pos = np.ascontiguousarray(g['adv_pos_in'].copy())
    spd = np.ones(len(pos), np.float32)
    dt, uin, max_age, seed, sx, scy, scz, shy, shz = g['adv_params']
    oracle_mod.advect(pos, spd, mac, solid, dims, dt, uin, max_age, int(seed), sx, scy, scz, shy, shz)
    assert np.array_equal(pos, g['adv_pos'])
    assert np.array_equal(spd, g['adv_spd'])
    q16, q8 = oracle_mod.pack(pos, spd, dims)
    assert np.array_equal(q16, g['pack_q16'])
    assert np.array_equal(q8, g['pack_q8'])
    for axis in (0, 1, 2):
        for field in range(4):
            a = g[f'slice_{axis}_{field}_args']
            out = oracle_mod.slice_(mac, solid, dims, int(a[0]), int(a[1]), int(a[2]), float(uin), float(a[3]),
                                    float(a[4]), float(a[5]))
            assert np.array_equal(out, g[f'slice_{axis}_{field}']), (axis, field)
    cp = oracle_mod.cp(mac, solid, np.ascontiguousarray(g['cp_verts']), np.ascontiguousarray(g['cp_norms']), dims,
                       float(uin))
    assert np.array_equal(cp, g['cp'])


def test_golden_fixture_covers_branches():
    """The fixtures actually exercise the rare branches they claim to."""
    g = golden('random_12x8x10_f32.npz')
    mac = g['mac_in']
    assert (mac[:, 3] < 0.9).any() and (mac[:, 3] > 1.1).any()
    assert (mac[:, 0] < 0).any()
    assert set(np.unique(g['solid'])) >= {0, 1, 2, 3}
    s = golden('sphere_32x16x16_f32.npz')
    pos_in, pos_out = s['adv_pos_in'], s['adv_pos']
    died = pos_out[:, 3] == 0
    assert died.any() and (~died).any()
