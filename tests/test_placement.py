"""Session placement over several GPUs (placement.py) on the CPU: the placement rule, the
merged statistics, and two gloo ranks serving one arrival stream with fake tunnels -- both
ranks compute the same placement with no exchange, and every session is served by exactly
one of them."""
import multiprocessing as mp
import socket
from datetime import timedelta

import numpy as np
import pytest

import placement
import serving


class _S:
    count = 0

    def __init__(self, n, lifetime=1e9):
        self.n, self.lifetime = n, lifetime
        self.id = _S.count
        _S.count += 1


def test_least_connected_cells_with_ties_to_lower_index():
    p = placement.Placer(3, 100, footprint=lambda s: s.n)
    assert [p.place(_S(10), 0.0) for _ in range(3)] == [0, 1, 2]
    assert p.place(_S(30), 1.0) == 0
    assert p.place(_S(5), 1.0) == 1
    assert p.place(_S(5), 1.0) == 2
    assert p.place(_S(1), 1.0) == 1        # gpu 1 and 2 both hold 15 cells; the lower index wins
    assert p.cells == [40, 16, 15]
    assert p.assignment == [0, 1, 2, 0, 1, 2, 1]


def test_budget_first_then_smallest_footprint():
    p = placement.Placer(2, 100, footprint=lambda s: 10 * s.n)
    assert p.place(_S(1), 0.0) == 0        # 10 bytes
    assert p.place(_S(9), 0.0) == 1        # 90 bytes
    assert p.place(_S(2), 0.0) == 0        # fewest cells and fits
    assert p.place(_S(5), 0.0) == 0        # 50 bytes fit only gpu 0 (30 + 50 <= 100)
    assert p.bytes == [80, 90]
    # 30 bytes fit nowhere: it waits on the GPU with the smaller footprint
    assert p.place(_S(3), 0.0) == 0
    assert p.bytes == [110, 90]


def test_departures_free_the_gpu():
    p = placement.Placer(2, 100, footprint=lambda s: s.n)
    assert p.place(_S(50, lifetime=1.0), 0.0) == 0
    assert p.place(_S(10, lifetime=5.0), 0.5) == 1
    assert p.place(_S(20), 0.9) == 1       # gpu 0 still holds 50 cells
    assert p.place(_S(20), 1.0) == 0       # its session has left at t = 1.0
    assert p.cells == [20, 30]
    with pytest.raises(ValueError):
        p.place(_S(1), 0.5)


def test_departures_reported_by_a_front_end():
    """Unknown lifetimes: sessions stay until leave() reports their client gone."""
    p = placement.Placer(2, 100, footprint=lambda s: s.n)
    a, b = _S(40, lifetime=float('inf')), _S(10, lifetime=float('inf'))
    assert p.place(a, 0.0) == 0 and p.place(b, 0.0) == 1
    assert p.place(_S(5, lifetime=float('inf')), 50.0) == 1  # a is still connected
    p.leave(a, 60.0)
    assert p.cells == [0, 15] and p.bytes == [0, 15]
    p.leave(a, 61.0)  # already gone: ignored
    assert p.place(_S(5, lifetime=float('inf')), 62.0) == 0
    with pytest.raises(ValueError):
        p.leave(b, 10.0)


def test_merge_pools_latencies_and_sums_counts():
    keys = dict(p50_ms=0, p99_ms=0, abandoned=0, retired=1, mean_active=2.5, glups=1.5, step_glups_device=2.0,
                peak_used_gb=3.0)
    a = dict(keys, frames=3, admitted=2, placed=2, failed=1)
    b = dict(keys, frames=1, admitted=1, placed=1, peak_used_gb=5.0, failed=0)
    m = placement.merge([a, b], [[0.001, 0.002, 0.003], [0.1]])
    assert m['frames'] == 4 and m['admitted'] == 3 and m['gpus'] == 2 and m['failed'] == 1
    assert m['glups'] == 3.0 and m['step_glups_device'] == 4.0 and m['mean_active'] == 5.0
    assert m['peak_used_gb_max'] == 5.0
    assert m['p50_ms'] == pytest.approx(np.percentile([1, 2, 3, 100], 50))
    assert m['max_ms'] == pytest.approx(100.0)
    assert [g['placed'] for g in m['per_gpu']] == [2, 1]


# ---- two gloo ranks, fake tunnels ----
class _FakeSolver:
    def __init__(self, s):
        self.num_p = s.particles
        self.last_forces6 = [0.0] * 6
        self.num_verts = 0

    def device_bytes(self):
        return 0

    def wait_event(self, e):
        pass

    def advance_particles(self, k, p):
        pass

    def launch_frame_packed(self, p, want_cp):
        pass

    def frame_ready(self):
        return True

    def collect_frame_packed(self, header):
        return b'frame'

    def synchronize(self):
        pass


class _FakeBatch:
    def __init__(self, solvers):
        pass

    def step(self, k):
        pass

    def event(self, timing=False):
        return None

    def close(self):
        pass


_MASKS = {size: [(None, 100.0)] for size in serving.SIZES}
_BUDGET = 12e9  # a few sessions per GPU, so some wait


def _rank(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group('gloo', init_method=f'tcp://127.0.0.1:{port}', rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    served = []

    def factory(device, **kw):
        srv = serving.SessionServer(device, solver_factory=_FakeSolver, batch_factory=lambda sv, p: _FakeBatch(sv),
                                    **kw)
        submit = srv.submit

        def record(s):
            served.append(s.id)
            submit(s)
        srv.submit = record
        return srv

    import lbm
    placer = placement.Placer(world, _BUDGET, lambda s: lbm.estimate_bytes(s.dims, 'fp32', s.particles))
    out, lat = placement.simulate_rank(rank, world, precision='fp32', budget=_BUDGET, particles=7,
                                       barrier=dist.barrier, placer=placer, duration=0.4, rate=40.0,
                                       mean_life=0.25, seed=3, device=None, mask_set=_MASKS,
                                       server_factory=factory)
    got = [None] * world
    dist.all_gather_object(got, (served, placer.assignment, out, lat))
    if rank == 0:
        q.put(got)
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def test_two_ranks_partition_one_arrival_stream():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=300)  # two spawned interpreters importing torch on a loaded host can be slow
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    served = [set(g[0]) for g in got]
    assign = [g[1] for g in got]
    common = min(len(a) for a in assign)
    assert common > 10
    # the same placement on both ranks, computed without any exchange
    assert assign[0][:common] == assign[1][:common]
    # every session of the common stream is served by exactly the rank it was placed on
    for sid in range(common):
        assert (sid in served[0]) + (sid in served[1]) == 1
        assert sid in served[assign[0][sid]]
    assert set(assign[0][:common]) == {0, 1}
    m = placement.merge([g[2] for g in got], [g[3] for g in got])
    assert m['frames'] == sum(len(g[3]) for g in got) > 0
    assert m['admitted'] == sum(g[2]['admitted'] for g in got)
