"""The reference server's own Engine, recorded driving a Solver over a real WebSocket
(tests/golden/engine_trace.npz, from server/app.py of the reference by make_engine_trace.py),
replayed on the library's CUDA Solver: the same calls in the same order with the same
arguments (the grid's Solver(dims, device) and reset, read-only mask and surface arrays as the
Engine decodes them from the client's gzip uploads, set_particles, step and frame with the
Engine's parameter dict), each frame packed as the Engine packs it.

Every frame must equal the one the reference server sent: the particle, slice and surface
pressure payloads byte for byte, the header field for field. The one tolerance is the forces
in the header: the reference sums them in float32 with atomics (server/lbm.py:194-197, here in
Warp's serial CPU order), the library in float64, so they agree to float32 rounding of the sum
(relative 1e-5 of the largest component)."""
import numpy as np
import pytest

import engine_replay

pytestmark = pytest.mark.gpu


def test_reference_engine_calls_on_the_cuda_solver_give_the_reference_frames():
    import wire
    from lbm import Solver
    events, frames, seed = engine_replay.load()
    got = engine_replay.replay(events, frames, lambda dims: Solver(dims, 'cuda:0', seed=seed))
    assert len(got) == len(frames)
    for j, (a, b) in enumerate(zip(got, frames)):
        da, db = wire.decode(a), wire.decode(b)
        ha, hb = dict(da['header']), dict(db['header'])
        fa, fb = np.array(ha.pop('forces')), np.array(hb.pop('forces'))
        assert ha == hb, f'frame {j}: header'
        np.testing.assert_allclose(fa, fb, rtol=0, atol=1e-5 * max(1e-6, float(np.abs(fb).max())),
                                   err_msg=f'frame {j}: forces')
        for part in ('parts16', 'parts8', 'slice', 'cp'):
            assert (part in da) == (part in db), f'frame {j}: {part} present in one only'
            if part in db:
                assert np.array_equal(da[part], db[part]), f'frame {j}: {part}'
