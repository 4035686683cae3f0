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
        self.launched = 0
        self.advanced = 0

    def device_bytes(self):
        return 0

    def wait_event(self, e):
        pass

    def advance_particles(self, k, p):
        self.advanced += k

    def launch_frame_packed(self, p, want_cp):
        self.launched += 1

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

    def step(self, k):
        assert not self.closed
        self.clock.t += sum(s.s.n for s in self.solvers) * k / self.rate

    def event(self, timing=False):
        return None

    def close(self):
        self.closed = True


def _server(clock, rate=1e12, budget=100.0):
    FakeBatch.log = []
    return serving.SessionServer(device=None, budget_bytes=budget, clock=clock, solver_factory=FakeSolver,
                                 batch_factory=lambda sv, p: FakeBatch(clock, rate, sv),
                                 footprint=lambda s: float(s.n))


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
