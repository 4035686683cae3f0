"""Serving loop on the GPU: every frame a session receives in the mix (sessions of different
sizes arriving, stepping together in one TunnelBatch and retiring at different rounds) is the
same, byte for byte, as the frame the same session gets when its tunnel runs alone through
Solver.step and the packed frame path. Batching is bit-exact, so the tolerance is zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


def _sessions():
    import bodies
    import serving
    specs = [((64, 24, 20), 0.05, 0.51, 1e9), ((48, 16, 16), 0.07, 0.53, 0.22), ((96, 32, 24), 0.04, 0.505, 1e9),
             ((40, 12, 14), 0.06, 0.52, 1e9)]
    out = []
    for k, (dims, uin, tau, life) in enumerate(specs):
        solid, _ = bodies.ellipsoid_union(dims, 2, 300 + k, scale=dims[0] / 256.0, floor='belt')
        out.append(serving.Session(k, dims, solid, dict(uIn=uin, tau=tau, smag=0.16), life, particles=200 + 50 * k))
    return out


def _alone(s, frames, precision, k):
    from lbm import Solver
    sv = Solver(s.dims, 'cuda:0', precision=precision, seed=s.id)
    sv.set_solid(s.solid)
    sv.reset(s.p['uIn'])
    sv.set_particles(s.particles, s.p)
    out = []
    for _ in range(frames):
        sv.step(k, s.p)
        sv.launch_frame_packed(s.p, False)
        header = dict(type='frame', dims=list(s.dims), numP=sv.num_p, numVerts=0, forces=None, steps=k, mlups=0.0,
                      running=True)
        out.append(sv.collect_frame_packed(header))
    return out


@pytest.mark.parametrize('mode', ['streams', 'persistent'])
@pytest.mark.parametrize('precision', ['fp32', 'fp16'])
def test_each_session_same_alone_and_in_the_mix(precision, mode):
    import serving
    clock = Clock()
    srv = serving.SessionServer('cuda:0', budget_bytes=1e9, precision=precision, clock=clock, keep_frames=True,
                                tile=2, batch_mode=mode)
    ss = _sessions()
    srv.submit(ss[0])
    srv.submit(ss[1])
    for r in range(9):
        clock.t = r * 0.05  # rounds further apart than the 1/30 s request period: all due
        if r == 2:
            srv.submit(ss[2])
        if r == 5:
            srv.submit(ss[3])
        srv.round()
    assert srv.retired == 1 and srv.admitted == 4
    assert srv.rebuilds == 3  # {0,1}, {0,1,2}, then {0,2,3} (1 retires as 3 joins, round 5)
    got = {}
    for sid, frame in srv.frame_log:
        got.setdefault(sid, []).append(frame)
    assert [len(got[i]) for i in range(4)] == [9, 5, 7, 4]
    for s in ss:
        ref = _alone(s, len(got[s.id]), precision, srv.steps_per_frame)
        for j, (a, b) in enumerate(zip(got[s.id], ref)):
            assert a == b, f'session {s.id} frame {j} differs from the session run alone'
    assert np.isfinite([s.cd for s in ss]).all()
    srv.close()
