"""Host logic of the serving loop (serving.SessionServer) with fake solvers, a fake batch and
a manual clock: FIFO admission against the HBM budget, abandonment, retirement, request
pacing, latency accounting and batch rebuilds only on membership changes."""
import pytest

import serving


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class FakeSolver:
    def __init__(self, s):
        self.s = s
        self.num_p = s.particles
        self.last_forces6 = [0.0] * 6
        self.num_verts = 0 if s.verts is None else len(s.verts)
        self.launched = 0
        self.advanced = 0
        self.calls = []
        self.cp_frames = []

    def set_particles(self, count, p):
        self.num_p = count
        self.calls.append(('set_particles', count))

    def reset(self, uin):
        self.calls.append(('reset', uin))

    def set_solid(self, solid):
        self.calls.append(('set_solid', bytes(solid)))

    def set_surface(self, verts, norms):
        self.num_verts = len(verts)
        self.calls.append(('set_surface', len(verts)))

    def device_bytes(self):
        return 0

    def wait_event(self, e):
        pass

    def advance_particles(self, k, p):
        self.advanced += k

    def launch_frame_packed(self, p, want_cp):
        self.launched += 1
        if want_cp:
            self.cp_frames.append(self.launched)

    def frame_ready(self):
        return True

    def collect_frame_packed(self, header):
        return repr((self.s.id, self.launched, sorted(header))).encode()

    def synchronize(self):
        pass


class FakeBatch:
    """Steps cost `cells * k / rate` seconds of the manual clock."""

    log = []

    def __init__(self, clock, rate, solvers):
        self.clock, self.rate, self.solvers = clock, rate, solvers
        self.closed = False
        FakeBatch.log.append(tuple(s.s.id for s in solvers))

    steps = []

    def step(self, k):
        assert not self.closed
        FakeBatch.steps.append(k)
        ks = k if isinstance(k, list) else [k] * len(self.solvers)
        self.clock.t += sum(s.s.n * kk for s, kk in zip(self.solvers, ks)) / self.rate

    def event(self, timing=False):
        return None

    def close(self):
        self.closed = True


def _server(clock, rate=1e12, budget=100.0, solver_factory=FakeSolver, **kw):
    FakeBatch.log = []
    FakeBatch.steps = []
    return serving.SessionServer(device=None, budget_bytes=budget, clock=clock, solver_factory=solver_factory,
                                 batch_factory=lambda sv, p: FakeBatch(clock, rate, sv),
                                 footprint=lambda s: float(s.n), **kw)


def _session(sid, n, life=1e9, arrival=0.0):
    return serving.Session(sid, (n, 1, 1), None, dict(uIn=0.05, tau=0.51, smag=0.16), life, particles=7,
                           frontal=1, arrival=arrival)


def test_fifo_admission_against_budget():
    c = Clock()
    srv = _server(c, budget=10)
    a, b, d = _session(0, 6, life=1.0), _session(1, 5), _session(2, 3)
    for s in (a, b, d):
        srv.submit(s)
    srv.round()
    assert list(srv.active) == [0] and [s.id for s in srv.queue] == [1, 2]  # no skipping past b
    assert srv.used == 6
    c.t = 1.0  # a's lifetime is over
    srv.round()
    assert list(srv.active) == [1, 2] and not srv.queue
    assert srv.retired == 1 and srv.used == 8 and srv.peak_used == 8
    assert FakeBatch.log == [(0,), (1, 2)]


def test_abandoned_while_queued():
    c = Clock()
    srv = _server(c, budget=5)
    srv.submit(_session(0, 5, life=2.0))
    srv.submit(_session(1, 5, life=1.5))
    srv.submit(_session(2, 1))
    srv.round()
    c.t = 1.6
    srv.round()
    assert srv.abandoned == 1 and [s.id for s in srv.queue] == [2]
    c.t = 2.0
    srv.round()
    assert list(srv.active) == [2] and srv.retired == 1


def test_pacing_at_fps_when_gpu_is_fast():
    c = Clock()
    srv = _server(c)
    for i in range(3):
        srv.submit(_session(i, 2))
    while c.t < 1.0:
        srv.round()
        c.t += 0.001
    s0 = srv.active[0]
    assert 29 <= s0.frames <= 31
    assert s0.solver.advanced == 10 * s0.frames
    assert max(srv.latencies) < 0.0011  # the fake GPU takes no time; the loop polls every 1 ms
    assert srv.rebuilds == 1  # the same three sessions every round


def test_oversubscribed_latency_is_round_time():
    c = Clock()
    rate = 1000.0  # cells*steps per second: 3 sessions x 20 cells x 10 steps = 0.6 s per round
    srv = _server(c, rate=rate)
    for i in range(3):
        srv.submit(_session(i, 20))
    for _ in range(5):
        srv.round()
    st = srv.stats()
    assert srv.rebuilds == 1 and st['frames'] == 15
    # first round: requested at 0, ready at 0.6; afterwards each request waits one round
    assert st['p50_ms'] == pytest.approx(600.0)
    assert srv.cell_updates / (c.t - srv.t0) == pytest.approx(rate)  # the fake GPU never idles
    slow = st['slow_rounds']  # the five rounds, longest first, then the median one
    assert len(slow) == 6 and slow[-1]['median'] and all(r['sessions'] == 3 for r in slow)
    assert [r['ms'] for r in slow[:5]] == sorted((r['ms'] for r in slow[:5]), reverse=True)
    assert slow[-1]['ms'] == pytest.approx(600.0)


def test_arrival_joins_next_round_and_batch_rebuilds():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 2))
    srv.round()
    srv.submit(_session(1, 2))
    c.t += 1 / 30
    srv.round()
    assert FakeBatch.log == [(0,), (0, 1)]
    assert srv.active[1].frames == 1 and srv.active[0].frames == 2


# ---- client commands (server/app.py:104-149, routed to the client's session) ----
def _upload(header, payload):
    import wire
    return wire.decode_upload(wire.encode_upload(header, payload))


def test_commands_run_at_the_next_round_in_order():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 4))
    srv.round()
    sv = srv.active[0].solver
    srv.command(0, {'type': 'params', 'uIn': 0.08, 'particles': 9})
    srv.command(0, {'type': 'reset'})
    srv.command(0, {'type': 'respawn'})
    assert sv.calls == []  # nothing before the round
    c.t += 1 / 30
    srv.round()
    assert sv.calls == [('set_particles', 9), ('reset', 0.08), ('set_particles', 9)]
    assert srv.active[0].p['uIn'] == 0.08
    assert FakeBatch.log == [(0,), (0,)]  # new flow parameters: the batch is rebuilt


def test_uploads_checked_like_the_engine():
    import numpy as np
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 4))  # dims (4, 1, 1)
    srv.round()
    sv = srv.active[0].solver
    good = np.array([0, 1, 2, 0], np.uint8)
    srv.command(0, *_upload({'type': 'solid', 'dims': [4, 1, 1]}, good.tobytes()))
    srv.command(0, *_upload({'type': 'solid', 'dims': [5, 1, 1]}, np.zeros(5, np.uint8).tobytes()))  # other grid
    srv.command(0, *_upload({'type': 'solid', 'dims': [4, 1, 1]}, np.zeros(3, np.uint8).tobytes()))  # short
    verts = np.arange(12, dtype=np.float32).reshape(2, 6)
    srv.command(0, *_upload({'type': 'surface', 'numVerts': 2}, verts.tobytes()))
    srv.command(0, *_upload({'type': 'surface', 'numVerts': 3}, verts.tobytes()))  # size mismatch
    c.t += 1 / 30
    srv.round()
    assert sv.calls == [('set_solid', good.tobytes()), ('set_surface', 2)]
    assert np.array_equal(srv.active[0].solid, good)
    with pytest.raises(ValueError):
        srv.command(0, {'type': 'grid', 'res': 'high'})


def test_queued_session_keeps_its_commands():
    import numpy as np
    c = Clock()
    srv = _server(c, budget=4)
    srv.submit(_session(0, 4, life=1.0))
    srv.submit(_session(1, 4))
    srv.round()
    srv.command(1, {'type': 'params', 'tau': 0.6})
    srv.command(1, *_upload({'type': 'solid', 'dims': [4, 1, 1]}, np.ones(4, np.uint8).tobytes()))
    srv.command(7, {'type': 'reset'})  # no such session: ignored
    c.t = 1.0
    srv.round()
    s1 = srv.active[1]
    assert s1.p['tau'] == 0.6 and np.array_equal(s1.solid, np.ones(4, np.uint8))
    assert s1.solver.calls == []  # created from the updated session, nothing replayed


def test_client_pacing_waits_for_ready():
    c = Clock()
    srv = _server(c, pacing='client')
    srv.submit(_session(0, 2))
    for _ in range(3):
        srv.round()
        c.t += 0.01
    assert srv.active[0].frames == 1
    assert srv.round_frames == []
    srv.command(0, {'type': 'ready'})
    srv.round()
    assert srv.active[0].frames == 2
    assert [sid for sid, _ in srv.round_frames] == [0]
    assert srv.latencies[-1] < 1e-6  # requested at the ack, served in the same round


def test_paused_session_is_not_stepped_and_frames_slow_down():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 2))
    srv.submit(_session(1, 2))
    srv.command(1, {'type': 'params', 'running': False})
    while c.t < 1.0:
        srv.round()
        c.t += 0.001
    a, b = srv.active[0], srv.active[1]
    assert a.solver.advanced == 10 * a.frames and b.solver.advanced == 0
    assert 29 <= a.frames <= 31 and 11 <= b.frames <= 13  # paused sessions at 12 Hz
    assert all(key == (0,) for key in FakeBatch.log)


def test_per_session_steps_with_the_streams_executor():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 2))
    srv.submit(_session(1, 2))
    srv.command(1, {'type': 'params', 'steps': 4})
    srv.round()
    assert FakeBatch.steps == [[10, 4]]
    assert srv.active[1].solver.advanced == 4
    # the parameter-space batched tiles (the default) step sessions by their own counts too
    q = _server(c, batch_mode='persistent')
    assert q.tile == 229 and q.steps_each
    q.submit(_session(0, 2))
    q.submit(_session(1, 2))
    q.command(1, {'type': 'params', 'steps': 4})
    q.round()
    assert FakeBatch.steps == [[10, 4]]
    p = _server(c, batch_mode='persistent', tile=103)
    p.submit(_session(0, 2))
    p.submit(_session(1, 2))
    p.command(1, {'type': 'params', 'steps': 4})
    p.round()
    assert FakeBatch.steps == [10]  # one launch of a work-list tile steps every tunnel alike


def test_surface_pressure_every_third_frame():
    import numpy as np
    c = Clock()
    srv = _server(c)
    s = _session(0, 2)
    s.p['cp'] = True
    srv.submit(s)
    srv.command(0, *_upload({'type': 'surface', 'numVerts': 1}, np.zeros(6, np.float32).tobytes()))
    for _ in range(7):
        srv.round()
        c.t += 1 / 30
    assert srv.active[0].solver.cp_frames == [3, 6]


# ---- failures stay with their session (server/app.py:115-122, 196-198) ----
def test_allocation_failure_is_reported_and_others_are_served():
    c = Clock()

    def factory(s):
        if s.id == 1:
            raise MemoryError('out of memory')
        return FakeSolver(s)
    srv = serving.SessionServer(device=None, budget_bytes=100, clock=c, solver_factory=factory,
                                batch_factory=lambda sv, p: FakeBatch(c, 1e12, sv), footprint=lambda s: float(s.n))
    for i in range(3):
        srv.submit(_session(i, 4))
    assert srv.round() == 2
    assert list(srv.active) == [0, 2] and srv.used == 8
    assert srv.failed == 1 and srv.errors[0][0] == 1 and 'Could not allocate 4x1x1 grid' in srv.errors[0][1]
    assert srv.stats()['failed'] == 1


def test_frame_failure_retires_only_that_session():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 4))
    srv.submit(_session(1, 4))
    srv.round()
    bad = srv.active[0].solver

    def boom(p, want_cp):
        raise RuntimeError('frame kernel failed')
    bad.launch_frame_packed = boom
    c.t += 1 / 30
    assert srv.round() == 1
    assert list(srv.active) == [1] and srv.used == 4 and srv.failed == 1
    assert srv.errors == [(0, "solver error: RuntimeError('frame kernel failed')")]
    c.t += 1 / 30
    srv.round()
    assert FakeBatch.log[-1] == (1,)  # rebuilt without the failed session
    assert srv.active[1].frames == 3


def test_one_tunnel_failing_in_a_step_fails_only_its_session():
    from batch import MemberError
    c = Clock()
    srv = _server(c)
    for i in range(3):
        srv.submit(_session(i, 2))
    orig = FakeBatch.step

    def step(self, k):
        orig(self, k)
        raise MemberError([(1, RuntimeError('bounded wait gave up'))])
    FakeBatch.step = step
    try:
        assert srv.round() == 2
    finally:
        FakeBatch.step = orig
    assert list(srv.active) == [0, 2] and srv.errors[0][0] == 1
    assert srv.active[0].frames == 1 and srv.active[2].frames == 1


def test_a_malformed_command_fails_alone():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 4))
    srv.round()
    srv.command(0, {'type': 'solid', 'dims': [4, 1, 1]}, b'not gzip')
    srv.command(0, {'type': 'params', 'tau': 0.55})
    c.t += 1 / 30
    assert srv.round() == 1
    assert srv.errors[0][0] == 0 and srv.errors[0][1].startswith('command failed:')
    assert srv.active[0].p['tau'] == 0.55  # the next command still ran


def test_disconnect_retires_or_dequeues():
    c = Clock()
    srv = _server(c, budget=4)
    srv.submit(_session(0, 4))
    srv.submit(_session(1, 4))
    srv.round()
    assert list(srv.active) == [0] and [q.id for q in srv.queue] == [1]
    srv.disconnect(1)  # still waiting: leaves the queue
    srv.disconnect(0)  # admitted: retired, memory released
    c.t += 1 / 30
    assert srv.round() == 0
    assert not srv.active and not srv.queue and srv.used == 0
    assert srv.retired == 1 and srv.abandoned == 1


def test_fits_is_the_admission_bound():
    c = Clock()
    srv = _server(c, budget=10)  # the fake footprint is one byte per cell
    assert srv.fits((10, 1, 1)) and not srv.fits((11, 1, 1))


def test_command_arriving_during_a_drain_waits_for_the_next_round():
    c = Clock()
    srv = _server(c)
    srv.submit(_session(0, 4))
    srv.round()
    sv = srv.active[0].solver
    orig = sv.reset

    def reset_and_more(uin):  # another thread's command lands while this round drains
        orig(uin)
        srv.command(0, {'type': 'respawn'})
    sv.reset = reset_and_more
    srv.command(0, {'type': 'reset'})
    c.t += 1 / 30
    srv.round()
    assert [k for k, _ in sv.calls] == ['reset']
    c.t += 1 / 30
    srv.round()
    assert [k for k, _ in sv.calls] == ['reset', 'set_particles']


def test_admission_worker_builds_tunnels_while_rounds_run():
    """With admit_thread the tunnels are built on a worker thread: a session joins the first
    round after its tunnel is ready, its memory is reserved from dispatch on, and commands sent
    while it is being built are applied, in order, once it is active."""
    import threading
    import time
    c = Clock()
    gate = threading.Event()

    def factory(s):
        if s.id == 1:
            raise MemoryError('out of memory')
        if s.id == 2:
            gate.wait(10)  # session 2's tunnel takes a while
        return FakeSolver(s)
    srv = serving.SessionServer(device=None, budget_bytes=100, clock=c, solver_factory=factory,
                                batch_factory=lambda sv, p: FakeBatch(c, 1e12, sv), footprint=lambda s: float(s.n),
                                admit_thread=True)
    try:
        for i in range(3):
            srv.submit(_session(i, 4))
        srv.round()
        assert srv.used == 12 and set(srv.building) <= {0, 1, 2}
        srv.command(2, {'type': 'params', 'tau': 0.7})
        srv.command(2, {'type': 'respawn'})
        for _ in range(200):  # session 0 is built at once, 1 fails, 2 waits for the gate
            c.t += 1 / 30
            srv.round()
            if 0 in srv.active and srv.failed:
                break
            time.sleep(0.005)
        assert 0 in srv.active and 2 in srv.building and srv.active[0].frames >= 1
        assert srv.failed == 1 and 'Could not allocate' in srv.errors[0][1] and srv.used == 8
        gate.set()
        for _ in range(200):
            c.t += 1 / 30
            srv.round()
            if 2 in srv.active:
                break
            time.sleep(0.005)
        s2 = srv.active[2]
        assert s2.p['tau'] == 0.7 and s2.solver.calls == [('set_particles', 7)]
    finally:
        gate.set()
        srv.close()


class RecyclingSolver(FakeSolver):
    made = 0

    def __init__(self, s):
        super().__init__(s)
        RecyclingSolver.made += 1
        self.recycled = 0

    def recycle(self, seed=None):
        self.recycled += 1


def _recycling_factory(s):
    sv = s.reuse
    if sv is None:
        return RecyclingSolver(s)
    s.reuse = None
    sv.recycle(s.id)
    sv.s = s
    return sv


def test_retired_tunnels_are_kept_and_reused_by_the_same_grid():
    c = Clock()
    RecyclingSolver.made = 0
    srv = _server(c, budget=20, solver_factory=_recycling_factory)
    a, b = _session(0, 6, life=1.0), _session(1, 4, life=1.0)
    srv.submit(a)
    srv.submit(b)
    srv.round()
    c.t = 1.0  # both retire; their tunnels are kept, still charged to the budget
    srv.round()
    assert srv.retired == 2 and srv.used == 0 and srv.pooled == 10 and a.solver is None
    d = _session(2, 6)  # the grid of session 0: takes its tunnel, no new solver
    srv.submit(d)
    srv.round()
    assert srv.pool_hits == 1 and RecyclingSolver.made == 2 and d.solver.recycled == 1
    assert srv.used == 6 and srv.pooled == 4
    e = _session(3, 12)  # another grid that needs the kept 4 bytes: the kept tunnel is dropped
    srv.submit(e)
    srv.round()
    assert srv.pool_evictions == 1 and srv.pooled == 0 and srv.used == 18 and RecyclingSolver.made == 3
    st = srv.stats()
    assert st['tunnels_reused'] == 1 and st['kept_tunnels_dropped'] == 1 and st['kept_gb_end'] == 0


def test_a_kept_tunnel_waits_when_memory_is_short_and_is_never_dropped_for_its_own_grid():
    c = Clock()
    srv = _server(c, budget=10, solver_factory=_recycling_factory)
    srv.submit(_session(0, 6, life=1.0))
    srv.submit(_session(1, 4))
    srv.round()
    c.t = 1.0
    srv.round()
    assert srv.pooled == 6 and srv.used == 4
    srv.submit(_session(2, 6))  # its grid's tunnel is kept: 4 + 6 fits exactly
    srv.round()
    assert srv.pool_hits == 1 and srv.pool_evictions == 0 and srv.used == 10 and srv.pooled == 0


def test_at_most_new_per_round_tunnels_are_allocated_each_round():
    c = Clock()
    RecyclingSolver.made = 0
    srv = _server(c, budget=100, solver_factory=_recycling_factory, new_per_round=1)
    srv.submit(_session(0, 4, life=1.0))
    srv.round()
    c.t = 1.0
    srv.round()  # session 0 retires; its tunnel is kept
    for i in (1, 2, 3):
        srv.submit(_session(i, 5 if i != 2 else 4))
    c.t = 1.1
    srv.round()  # 1 is this round's allocation; 2 takes the kept tunnel (not counted); 3 waits
    assert list(srv.active) == [1, 2] and [s.id for s in srv.queue] == [3]
    assert RecyclingSolver.made == 2 and srv.pool_hits == 1
    c.t = 1.2
    srv.round()  # the next round allocates 3
    assert list(srv.active) == [1, 2, 3] and RecyclingSolver.made == 3


def test_arena_ranges_follow_the_tunnels_and_an_arrival_waits_for_a_range():
    import arena
    c = Clock()
    unit = 256

    def factory(s):  # the default factory's arena use, with fake tunnels
        if s.reuse is not None:
            sv, s.reuse = s.reuse, None
            sv.recycle(s.id)
            sv.s = s
            return sv
        off = srv._arena.alloc(s.n * unit)
        assert off is not None
        sv = RecyclingSolver(s)
        sv.arena_off = off
        return sv

    srv = _server(c, budget=100, solver_factory=factory, arena=True)
    srv._arena = arena.Arena(10 * unit)
    srv._state_bytes = lambda s: s.n * unit
    srv._allocate = lambda s: None  # marks the default path; admission here builds in the round
    a, b, d = _session(0, 4, life=1.0), _session(1, 4), _session(2, 3)
    for s in (a, b, d):
        srv.submit(s)
    srv.round()
    # the budget (100) has room for the third, the arena (2 units free) has not
    assert list(srv.active) == [0, 1] and [s.id for s in srv.queue] == [2] and srv.arena_waits == 1
    c.t = 1.0  # session 0 retires and its tunnel is kept; then session 2, of another grid, needs
    srv.round()  # a range: the kept tunnel is dropped and its range reused
    assert list(srv.active) == [1, 2] and srv.pool_evictions == 1 and srv.pooled == 0
    assert srv._arena.used == {0: 3 * unit, 4 * unit: 4 * unit}
    c.t = 2.0
    srv.disconnect(1)
    srv.disconnect(2)
    srv.round()
    srv.close()
