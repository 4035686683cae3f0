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


EXECUTORS = [('streams', 0), ('persistent', 2), ('persistent', 229)]


@pytest.mark.parametrize('mode,tile', EXECUTORS)
@pytest.mark.parametrize('precision', ['fp32', 'fp16'])
def test_each_session_same_alone_and_in_the_mix(precision, mode, tile):
    import serving
    clock = Clock()
    srv = serving.SessionServer('cuda:0', budget_bytes=1e9, precision=precision, clock=clock, keep_frames=True,
                                tile=tile, batch_mode=mode, rate_in_header=False)
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


def _engine_replay(s0, script, precision, each, rounds):
    """One session alone, driven as the reference Engine drives its Solver (server/app.py:
    104-193): commands, then step(steps) when running, then a frame (Cp every third frame).
    each: the session's own 'steps' per frame (else the server's 10)."""
    import gzip
    import numpy as np
    import wire
    from lbm import Solver
    p = dict(s0.p)
    sv = Solver(s0.dims, 'cuda:0', precision=precision, seed=s0.id)
    sv.set_solid(s0.solid)
    sv.reset(p['uIn'])
    sv.set_particles(s0.particles, p)
    particles = s0.particles
    frames, frame_no = [], 0
    for r in range(rounds):
        for msg, payload in script.get((r, s0.id), []):
            t = msg['type']
            if t == 'params':
                old = int(p.get('particles', particles))
                p.update({k: v for k, v in msg.items() if k != 'type'})
                new = int(p.get('particles', old))
                if new != old:
                    particles = new
                    if sv.num_p:
                        sv.set_particles(new, p)
            elif t == 'reset':
                sv.reset(p['uIn'])
            elif t == 'respawn':
                sv.set_particles(int(p.get('particles', particles)), p)
            else:
                got = wire.upload_arrays(msg, payload, s0.dims)
                if got[0] == 'solid':
                    sv.set_solid(got[1])
                else:
                    sv.set_surface(got[1], got[2])
        running = bool(p.get('running', True))
        k = (int(p.get('steps', 10)) if each else 10) if running else 0
        if k:
            sv.step(k, p)
        frame_no += 1
        every = max(3, sv.num_verts // 20000)
        want_cp = bool(p.get('cp')) and sv.num_verts > 0 and frame_no % every == 0
        sv.launch_frame_packed(p, want_cp)
        header = dict(type='frame', dims=list(s0.dims), numP=sv.num_p, numVerts=sv.num_verts, forces=None, steps=k,
                      mlups=0.0, running=running)
        frames.append(sv.collect_frame_packed(header))
    return frames


@pytest.mark.parametrize('mode,tile', EXECUTORS)
def test_client_commands_match_the_engine_semantics(mode, tile):
    """Two sessions under client pacing receive parameter changes, a reset, a respawn, a mask
    and a surface upload, a pause and a resume, through SessionServer.command; every frame
    equals the frame the same session gets alone when the same commands are applied the way
    the reference's Engine applies them."""
    import copy
    import numpy as np
    import bodies
    import serving
    import wire
    ss = _sessions()[:2]
    for s in ss:
        s.lifetime = 1e9
    originals = [copy.deepcopy(s) for s in ss]
    new_solid, _ = bodies.ellipsoid_union(ss[1].dims, 3, 977, scale=ss[1].dims[0] / 256.0, floor='belt')
    verts, norms = bodies.surface_points(ss[0].solid, ss[0].dims)
    surf = np.concatenate([verts.reshape(-1), norms.reshape(-1)]).astype(np.float32).tobytes()
    up = lambda h, b: wire.decode_upload(wire.encode_upload(h, b))
    script = {
        (1, 0): [({'type': 'params', 'uIn': 0.065, 'steps': 6, 'cp': True}, None),
                 up({'type': 'surface', 'numVerts': len(verts)}, surf)],
        (1, 1): [up({'type': 'solid', 'dims': list(ss[1].dims)}, new_solid.tobytes())],
        (2, 0): [({'type': 'reset'}, None), ({'type': 'respawn'}, None)],
        (2, 1): [({'type': 'params', 'running': False}, None)],
        (4, 1): [({'type': 'params', 'running': True, 'particles': 120}, None)],
        (5, 0): [({'type': 'params', 'tau': 0.56}, None)],
    }
    rounds = 7
    clock = Clock()
    srv = serving.SessionServer('cuda:0', budget_bytes=1e9, precision='fp32', clock=clock, keep_frames=True,
                                tile=tile, batch_mode=mode, pacing='client', rate_in_header=False)
    for s in ss:
        srv.submit(s)
    for r in range(rounds):
        clock.t = r * 0.1
        for sid in (0, 1):
            if r:
                srv.command(sid, {'type': 'ready'})
            for msg, payload in script.get((r, sid), []):
                srv.command(sid, msg, payload)
        assert srv.round() == 2
    got = {0: [], 1: []}
    for sid, frame in srv.frame_log:
        got[sid].append(frame)
    srv.close()
    for s0 in originals:
        want = _engine_replay(s0, script, 'fp32', srv.steps_each, rounds)
        assert len(got[s0.id]) == rounds
        for r, (a, b) in enumerate(zip(got[s0.id], want)):
            assert a == b, f'session {s0.id} frame {r}'


@pytest.mark.parametrize('precision', ['fp32', 'fp16'])
def test_recycled_tunnel_equals_a_new_one(precision):
    """A Solver that served one session (surface, particles, frames with Cp, an odd step count)
    and is then recycled gives the next session the frames and populations a new Solver gives."""
    import bodies
    import serving
    from lbm import Solver
    dims = (64, 24, 20)
    first = _sessions()[0]
    second = serving.Session(7, dims, bodies.ellipsoid_union(dims, 3, 977, scale=dims[0] / 256.0, floor='belt')[0],
                             dict(uIn=0.06, tau=0.52, smag=0.16), 1e9, particles=150)
    verts, norms = bodies.surface_points(first.solid, dims)

    def frames(sv, s, n, k, cp):
        out = []
        for _ in range(n):
            sv.step(k, s.p)
            sv.advance_particles(k, s.p)
            sv.launch_frame_packed(s.p, cp)
            header = dict(type='frame', dims=list(dims), numP=sv.num_p, numVerts=sv.num_verts, forces=None, steps=k,
                          mlups=0.0, running=True)
            out.append(sv.collect_frame_packed(header))
        return out

    used = Solver(dims, 'cuda:0', precision=precision, seed=first.id)
    used.set_solid(first.solid)
    used.set_surface(verts, norms)
    used.reset(first.p['uIn'])
    used.set_particles(first.particles, first.p)
    frames(used, first, 3, 7, True)
    used.recycle(seed=second.id)
    fresh = Solver(dims, 'cuda:0', precision=precision, seed=second.id)
    got = {}
    for name, sv in (('recycled', used), ('new', fresh)):
        sv.set_solid(second.solid)
        sv.reset(second.p['uIn'])
        sv.set_particles(second.particles, second.p)
        got[name] = (frames(sv, second, 4, 10, False), sv.populations(), sv.macro())
    assert got['recycled'][0] == got['new'][0]
    assert np.array_equal(got['recycled'][1], got['new'][1])
    assert np.array_equal(got['recycled'][2], got['new'][2])


@pytest.mark.parametrize('precision', ['fp32', 'fp16'])
def test_solver_on_arena_storage_equals_a_plain_one(precision):
    """A Solver whose per-cell state is a range of the serving arena (filled with garbage first,
    next to another dirty range) gives the frames and populations of a Solver that allocated
    its own."""
    import arena
    import lbm
    s0 = _sessions()[2]
    _, total = lbm.state_layout(s0.dims, precision)
    a = arena.Arena(3 * total + 4096, 'cuda:0')
    other, off = a.alloc(total), a.alloc(total)
    a.view(other, total).fill_(0x5a)
    a.view(off, total).fill_(0xa5)

    def run(sv):
        sv.set_solid(s0.solid)
        sv.reset(s0.p['uIn'])
        sv.set_particles(s0.particles, s0.p)
        out = []
        for _ in range(3):
            sv.step(7, s0.p)
            sv.advance_particles(7, s0.p)
            sv.launch_frame_packed(s0.p, False)
            header = dict(type='frame', dims=list(s0.dims), numP=sv.num_p, numVerts=0, forces=None, steps=7,
                          mlups=0.0, running=True)
            out.append(sv.collect_frame_packed(header))
        return out, sv.populations(), sv.macro()

    on_arena = run(lbm.Solver(s0.dims, 'cuda:0', precision=precision, seed=s0.id, storage=a.view(off, total)))
    plain = run(lbm.Solver(s0.dims, 'cuda:0', precision=precision, seed=s0.id))
    assert on_arena[0] == plain[0]
    assert np.array_equal(on_arena[1], plain[1]) and np.array_equal(on_arena[2], plain[2])
    assert bool((a.view(other, total) == 0x5a).all())  # the neighbouring range is untouched
