"""Device-assembled wire frames (Solver.launch_frame_packed / collect_frame_packed): the
frame bytes must equal the reference's packing (server/app.py:23-41, restated in wire.pack
and pinned to its output in test_wire.py) of the parts that Solver.frame() returns for the
same state, and decode as the browser client does (web/js/net.js:18-29)."""
import numpy as np
import pytest

import wire

pytestmark = pytest.mark.gpu

ORDER = ('type', 'dims', 'numP', 'numVerts', 'forces', 'steps', 'mlups', 'running')


def _solver(precision, particles, surface):
    import bodies
    from lbm import Solver
    dims = (64, 28, 36)
    solid = bodies.sphere_tunnel(dims, (20, 12, 18), 6.0, floor='belt')
    p = dict(uIn=0.08, tau=0.52, smag=0.16, maxAge=400.0, lref=12.0, seedX=2.0, seedCy=13.5, seedCz=17.5,
             seedHy=10.0, seedHz=10.0, slice=dict(axis=1, index=14, field=0, vmin=0.0, vmax=1.6))
    s = Solver(dims, 'cuda:0', precision=precision, seed=3)
    s.set_solid(solid)
    s.reset(p['uIn'])
    if surface:
        verts, norms = bodies.surface_points(solid, dims, max_points=777)
        s.set_surface(verts, norms)
    if particles:
        s.set_particles(particles, p)
    s.step(30, p)
    return s, p


def _reference_bytes(s, p, want_cp, steps=30):
    out = s.frame(p, want_cp)
    header = dict(type='frame', dims=[s.nx, s.ny, s.nz], numP=s.num_p, numVerts=s.num_verts,
                  forces=out['forces'], steps=steps, mlups=123.5, running=True)
    if 'slice' in out:
        header.update(sliceW=out['sliceW'], sliceH=out['sliceH'], sliceAxis=out['sliceAxis'])
    parts = [(k, out[k]) for k in wire.PART_ORDER if k in out]
    return wire.pack(header, parts), out


@pytest.mark.parametrize('precision', ['fp32', 'fp16'])
@pytest.mark.parametrize('particles,surface,want_cp,field', [
    (500, True, True, 0), (0, True, True, 2), (37, False, False, 1), (0, False, False, -1), (5000, True, False, 3)])
def test_packed_frame_equals_reference_pack(precision, particles, surface, want_cp, field):
    s, p = _solver(precision, particles, surface)
    p['slice']['field'] = field
    ref, out = _reference_bytes(s, p, want_cp)
    header = {k: None for k in ORDER}
    header.update(type='frame', dims=[s.nx, s.ny, s.nz], numP=s.num_p, numVerts=s.num_verts, steps=30,
                  mlups=123.5, running=True)
    for _ in range(2):  # the second call reuses the buffers
        s.launch_frame_packed(p, want_cp)
        got = s.collect_frame_packed(header)
        assert got == ref
        assert np.array_equal(s.last_forces6[:3], np.array(out['forces']))
    d = wire.decode(got)
    for k in wire.PART_ORDER:
        assert (k in d) == (k in out)
        if k in out:
            assert np.array_equal(d[k], out[k].view(wire.PART_DTYPE[k]))


def test_packed_frame_follows_steps():
    """Frames between steps track the state: each equals the unpacked path at that step."""
    s, p = _solver('fp32', 300, True)
    header = dict(type='frame', dims=[s.nx, s.ny, s.nz], numP=s.num_p, numVerts=s.num_verts, forces=None,
                  steps=10, mlups=123.5, running=True)
    seen = set()
    for _ in range(3):
        s.step(10, p)
        ref, _ = _reference_bytes(s, p, True, steps=10)
        s.launch_frame_packed(p, True)
        got = s.collect_frame_packed(header)
        assert got == ref
        seen.add(got)
    assert len(seen) == 3
