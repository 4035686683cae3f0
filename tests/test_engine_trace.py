"""The recorded reference Engine (tests/golden/engine_trace.npz, made by make_engine_trace.py
from the reference's own server/app.py) replayed on the oracle-backed stand-in Solver gives
back the recorded frames byte for byte: the fixture is what the reference server sends for
that client session, and the replay reproduces the Engine's packing. The CUDA Solver is
replayed against the same frames in test_gpu_engine_trace.py."""
import engine_replay


def test_fixture_frames_decode_as_the_browser_decodes():
    import wire
    events, frames, _ = engine_replay.load()
    assert len(frames) == 8 and sum(ev['method'] == 'frame' for ev in events) == 8
    kinds = set()
    for f in frames:
        d = wire.decode(f)
        kinds |= set(d['header']['offsets'])
    assert kinds == {'parts16', 'parts8', 'slice', 'cp'}
    assert {ev['method'] for ev in events} == {'init', 'reset', 'set_solid', 'set_surface', 'set_particles', 'step',
                                              'frame'}


def test_replay_on_the_oracle_reproduces_the_reference_server_frames(oracle_mod):
    from engine_solver import OracleSolver
    events, frames, seed = engine_replay.load()
    OracleSolver.seed_for_particles = seed
    got = engine_replay.replay(events, frames, lambda dims: OracleSolver(dims))
    assert len(got) == len(frames)
    for j, (a, b) in enumerate(zip(got, frames)):
        assert a == b, f'frame {j}'
