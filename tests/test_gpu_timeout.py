"""Failure detection without a GPU fault: the streaming step kernel waits on its copy
pipeline with a bounded wait. The test entry point wt_step_test_skip_chunk makes one chunk's
copies never start, so that wait runs out; the kernel must report WT_ERR_TIMEOUT through the tunnel's status word,
return on its own, and leave the context usable (a reset and normal steps then match the
oracle again)."""
import numpy as np
import pytest

import wtlib as W

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(oracle_mod):
    from lbm import Solver
    dims = (64, 20, 12)
    s = Solver(dims, 'cuda:0')
    s.reset(0.05)
    stream_tiles = [t[0] for t in W.step_tiles(W.F32) if t[1] < 0]
    s.set_tile(stream_tiles[0])
    p = dict(uIn=0.05, tau=0.51, smag=0.16)
    # chunk 0 is never loaded (the test-only entry point's hook)
    W.call('wt_step_test_skip_chunk', s.gp, s.cur, 1, p['uIn'], p['tau'], p['smag'], 0, 1, s.sh)
    s.cur ^= 1
    assert s.status() == W.WT_ERR_TIMEOUT
    s.reset(0.05)
    s.cur = 0
    s.step(4, p)
    assert s.status() == 0
    L = oracle_mod.Lattice(dims, oracle_mod.F32)
    L.reset(0.05)
    L.step(4, 0.05, 0.51, 0.16)
    assert np.array_equal(s.populations(), L.populations())
