"""The reference Solver's API over the CPU oracle, recording every call -- TEST INFRASTRUCTURE.

``OracleSolver`` has the methods and attributes the reference Engine drives
(``server/lbm.py:398-482``: ``Solver(dims, device)``, ``reset``, ``set_solid``, ``set_surface``,
``set_particles``, ``step``, ``slice_dims``, ``frame``; ``nx, ny, nz, n, num_p, num_verts``) and
computes each with the oracle, which equals the reference kernels bit for bit (golden vectors
in tests/golden). It exists so the reference's own server (``server/app.py``) can be run on a
machine without Warp or a GPU (tests/golden/make_engine_trace.py), and so the call sequence
its Engine issues can be recorded and replayed on the library's CUDA Solver.

Two choices the reference leaves open are fixed here the way the library's Solver fixes them:
``set_particles`` draws from ``numpy.random.default_rng(seed)`` (the reference's generator is
unseeded, server/lbm.py:430) and particle respawn uses the library's counter-based RNG (the
reference's Warp RNG is not available, server/lbm.py:256-259). Forces are the oracle's float
sums in the reference's serial order, as Warp's CPU backend forms them (server/lbm.py:194-197).

Every call is appended to ``trace`` as ``(method, args)`` with arrays copied, so that a replay
can issue the same calls in the same order.
"""
import numpy as np

import oracle

CP_RANGE = 1.2  # server/lbm.py:395


class OracleSolver:
    """Drop-in for the reference Solver, computed by the oracle. ``seed`` seeds set_particles."""

    seed_for_particles = 7
    instances = []  # every solver made (the recorder reads their traces)

    def __init__(self, dims, device=None):
        self.nx, self.ny, self.nz = (int(d) for d in dims)
        self.n = self.nx * self.ny * self.nz
        self.L = oracle.Lattice((self.nx, self.ny, self.nz), oracle.F32)
        self.num_p = 0
        self.num_verts = 0
        self.seed = 1
        self.rng = np.random.default_rng(self.seed_for_particles)
        self.trace = [('init', {'dims': [self.nx, self.ny, self.nz]})]
        OracleSolver.instances.append(self)

    def reset(self, uin):
        self.trace.append(('reset', {'uin': float(uin)}))
        self.L.reset(float(uin))

    def set_solid(self, arr):
        assert arr.size == self.n
        self.trace.append(('set_solid', {'solid': np.array(arr, np.uint8).copy()}))
        self.L.solid[:] = np.asarray(arr, np.uint8).reshape(-1)

    def set_surface(self, verts, norms):
        self.verts = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
        self.norms = np.ascontiguousarray(norms, np.float32).reshape(-1, 3)
        self.num_verts = len(self.verts)
        self.trace.append(('set_surface', {'verts': self.verts.copy(), 'norms': self.norms.copy()}))

    def set_particles(self, count, p):
        self.trace.append(('set_particles', {'count': int(count), 'p': _plain(p)}))
        rng = self.rng
        d = np.zeros((count, 4), np.float32)
        d[:, 0] = 2 + rng.random(count) * (self.nx - 8)
        d[:, 1] = p['seedCy'] + (rng.random(count) * 2 - 1) * p['seedHy']
        d[:, 2] = p['seedCz'] + (rng.random(count) * 2 - 1) * p['seedHz']
        d[:, 3] = rng.random(count) * p['maxAge'] * 0.5
        self.num_p = count
        self.pos = d
        self.spd = np.ones(count, np.float32)

    def step(self, steps, p):
        self.trace.append(('step', {'steps': int(steps), 'p': _plain(p)}))
        self.L.step(int(steps), p['uIn'], p['tau'], p['smag'])
        if self.num_p and steps:
            self.seed += 1
            oracle.advect(self.pos, self.spd, self.L.mac, self.L.solid, (self.nx, self.ny, self.nz), float(steps),
                          p['uIn'], p['maxAge'], self.seed, p['seedX'], p['seedCy'], p['seedCz'], p['seedHy'],
                          p['seedHz'])

    def slice_dims(self, axis):
        return {2: (self.nx, self.ny), 1: (self.nx, self.nz), 0: (self.nz, self.ny)}[axis]

    def frame(self, p, want_cp):
        self.trace.append(('frame', {'p': _plain(p), 'want_cp': bool(want_cp)}))
        dims = (self.nx, self.ny, self.nz)
        out = {}
        if self.num_p:
            out['parts16'], out['parts8'] = oracle.pack(self.pos, self.spd, dims)
        sl = p.get('slice')
        if sl and sl.get('field', -1) >= 0:
            axis = int(sl['axis'])
            w, h = self.slice_dims(axis)
            index = max(0, min(dims[axis] - 1, int(sl['index'])))
            out['slice'] = oracle.slice_(self.L.mac, self.L.solid, dims, axis, index, int(sl['field']), p['uIn'],
                                         p['lref'], float(sl['vmin']), float(sl['vmax']))
            out['sliceW'], out['sliceH'], out['sliceAxis'] = w, h, axis
        if want_cp and self.num_verts:
            out['cp'] = oracle.cp(self.L.mac, self.L.solid, self.verts, self.norms, dims, p['uIn'])
        ref, _, _ = self.L.forces()
        out['forces'] = [float(v) for v in ref]
        return out


def _plain(p):
    """A JSON-able copy of the Engine's parameter dict."""
    return {k: (dict(v) if isinstance(v, dict) else v) for k, v in p.items()}
