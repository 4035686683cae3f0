"""Many tunnels in one batch (wt_batch_*): each tunnel's populations must equal, bit for bit,
the same tunnel stepped alone with wt_step, for direct steps, odd step counts and CUDA-graph
replays."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tunnels(collision='exact', precision='fp32'):
    import bodies
    from lbm import Solver
    specs = [((64, 24, 20), 0.05, 0.51), ((48, 16, 16), 0.07, 0.53), ((96, 32, 24), 0.04, 0.505)]
    out = []
    for k, (dims, uin, tau) in enumerate(specs):
        solid, _ = bodies.ellipsoid_union(dims, 2, 100 + k, scale=dims[0] / 256.0, floor='belt')
        p = dict(uIn=uin, tau=tau, smag=0.16)
        s = Solver(dims, 'cuda:0', precision=precision, collision=collision)
        s.set_solid(solid)
        s.reset(uin)
        out.append((s, solid, p))
    return out


def _alone(dims, solid, p, steps, collision, precision):
    from lbm import Solver
    s = Solver(dims, 'cuda:0', precision=precision, collision=collision)
    s.set_solid(solid)
    s.reset(p['uIn'])
    s.step(steps, p)
    return s.populations(), s.macro()


@pytest.mark.parametrize('collision,precision', [('exact', 'fp32'), ('fast', 'fp16')])
@pytest.mark.parametrize('tile', [2, 3, 102, 118, 203, 218, 229])
def test_batch_equals_tunnels_alone(collision, precision, tile):
    from batch import TunnelBatch
    tun = _tunnels(collision, precision)
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], tile=tile)
    b.step(3)
    b.step(4)
    b.synchronize()
    for s, solid, p in tun:
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, 7, collision, precision)
        assert s.cur == 1
        assert np.array_equal(s.populations(), f)
        assert np.array_equal(s.macro(), mac)
    b.close()


def test_batch_graph_replay_equals_steps():
    from batch import TunnelBatch
    tun = _tunnels()
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], tile=2)
    b.capture(10)
    b.replay()
    b.replay()
    b.synchronize()
    for s, solid, p in tun:
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, 20, 'exact', 'fp32')
        assert s.cur == 0
        assert np.array_equal(s.populations(), f)
        assert np.array_equal(s.macro(), mac)
    b.close()


@pytest.mark.parametrize('collision,precision', [('exact', 'fp32'), ('fast', 'fp16')])
def test_streams_executor_equals_tunnels_alone(collision, precision):
    """mode='streams': every tunnel stepped by its own kernel on its own stream, at once."""
    from batch import TunnelBatch
    tun = _tunnels(collision, precision)
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], mode='streams')
    b.step(3)
    b.step(4)
    b.event().synchronize()
    for s, solid, p in tun:
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, 7, collision, precision)
        assert s.cur == 1
        assert np.array_equal(s.populations(), f)
        assert np.array_equal(s.macro(), mac)
    b.close()


def test_streams_executor_graph_replay_equals_steps():
    from batch import TunnelBatch
    tun = _tunnels('fast', 'fp16')
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], mode='streams')
    b.capture(10)
    b.replay()
    b.replay()
    b.event().synchronize()
    for s, solid, p in tun:
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, 20, 'fast', 'fp16')
        assert s.cur == 0
        assert np.array_equal(s.populations(), f)
        assert np.array_equal(s.macro(), mac)
    b.close()



@pytest.mark.parametrize('collision,precision', [('exact', 'fp32'), ('fast', 'fp16')])
def test_parameter_space_batch_steps_each_tunnel_by_its_own_count(collision, precision):
    """Tile 229 (descriptors in the kernel parameters) with uneven counts, one tunnel left as it
    is, then a graph replay: each tunnel equals itself stepped alone by its total."""
    from batch import TunnelBatch
    tun = _tunnels(collision, precision)
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], tile=229)
    b.step([3, 0, 5])
    b.step([2, 4, 1])
    b.capture(4)
    b.replay()
    b.synchronize()
    for (s, solid, p), k in zip(tun, [9, 8, 10]):
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, k, collision, precision)
        assert s.cur == k % 2
        assert np.array_equal(s.populations(), f)
        assert np.array_equal(s.macro(), mac)
    b.close()


def test_parameter_space_batch_launches_groups_of_tunnels():
    """More tunnels than one launch's parameter space holds (38 fp32 descriptors): the batch
    runs in groups, and every tunnel still equals itself alone."""
    import bodies
    from batch import TunnelBatch
    from lbm import Solver
    tun = []
    for k in range(41):
        dims = (16 + 2 * (k % 5), 8 + k % 3, 6 + k % 4)
        solid, _ = bodies.ellipsoid_union(dims, 1, 300 + k, scale=dims[0] / 128.0, floor='belt')
        p = dict(uIn=0.04 + 0.001 * k, tau=0.52, smag=0.16)
        s = Solver(dims, 'cuda:0')
        s.set_solid(solid)
        s.reset(p['uIn'])
        tun.append((s, solid, p))
    b = TunnelBatch([t[0] for t in tun], [t[2] for t in tun], tile=229)
    b.step([1 + k % 3 for k in range(41)])
    b.synchronize()
    for k, (s, solid, p) in enumerate(tun):
        f, mac = _alone((s.nx, s.ny, s.nz), solid, p, 1 + k % 3, 'exact', 'fp32')
        assert np.array_equal(s.populations(), f), f'tunnel {k}'
        assert np.array_equal(s.macro(), mac), f'tunnel {k}'
    b.close()
