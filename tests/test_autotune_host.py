"""The autotuner's selection logic with a fake tunnel and fake CUDA events (no GPU): repeats
interleaved across tiles, ranking by the median, and the sustained run-off of the finalists,
which must pick the tile that is fastest in long windows even when short windows rank another
tile first."""
import pytest

import autotune


class FakeClock:
    t = 0.0


class FakeEvent:
    def __init__(self, enable_timing=True):
        self.t = None

    def record(self, stream=None):
        self.t = FakeClock.t

    def synchronize(self):
        pass

    def elapsed_time(self, other):
        return other.t - self.t


class FakeSolver:
    """Per-step ms by tile: `short` in windows under 50 steps, `long` from 50 steps on (tile 18
    is the fastest in short windows and loses in long ones, as under a power cap)."""
    stream = None
    dev = None
    short = {3: 0.95, 18: 0.85, 30: 0.90, 34: 0.87, 35: 0.88, 12: 1.10}
    long = {3: 0.96, 18: 0.93, 30: 0.90, 34: 0.86, 35: 0.87, 12: 1.10}

    def __init__(self):
        self.tile = 0
        self.log = []

    def set_tile(self, t):
        self.tile = t

    def step(self, k, p):
        self.log.append((self.tile, k))
        if self.tile:
            FakeClock.t += k * (self.long if k >= 50 else self.short)[self.tile]


def _tune(monkeypatch, **kw):
    monkeypatch.setattr(autotune.torch.cuda, 'Event', FakeEvent)
    monkeypatch.setattr(autotune, 'admissible', lambda s: [(t, 2, 128, 8) for t in FakeSolver.short])
    monkeypatch.setattr(autotune, '_key', lambda s: 'fake')
    monkeypatch.setattr(autotune, '_save_file', lambda: None)
    s = FakeSolver()
    return s, autotune.tune(s, {}, force=True, **kw)


def test_screen_alone_picks_the_short_window_winner(monkeypatch):
    s, (tile, ms) = _tune(monkeypatch)
    assert tile == 18 and ms[18] == pytest.approx(0.85) and s.tile == 18
    # repeats interleaved: every tile is timed once before any tile is timed again
    timed = [t for t, k in s.log if k == 8]
    n = len(FakeSolver.short)
    assert timed[:n] == timed[n:2 * n] == list(FakeSolver.short)


def test_sustained_run_off_picks_the_long_window_winner(monkeypatch):
    s, (tile, ms) = _tune(monkeypatch, finalists=4)
    assert tile == 34 and s.tile == 34
    # the four fastest of the screen ran off in 100-step windows; the rest keep screen figures
    assert {t for t, k in s.log if k == 100} == {18, 34, 35, 30}
    assert ms[18] == pytest.approx(0.93) and ms[34] == pytest.approx(0.86) and ms[3] == pytest.approx(0.95)
