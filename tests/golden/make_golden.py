"""Generate golden vectors from the reference solver's OWN kernel code.

Runs ``server/lbm.py`` of RICKxxROLLING/wind-tunnel under the stub-``warp`` shim
(``oracle/warp_shim.py``): the generated ``init_kernel``/``step_kernel``/``force_kernel``
text and the hand-written ``advect_kernel``/``pack_particles``/``slice_kernel``/
``cp_kernel`` execute serially in tid order (Warp's CPU order) with numpy float32 (and
float64) scalars. The outputs are written as small ``.npz`` fixtures beside this script;
tests pin the C++ oracle and the CUDA kernels to them.

Usage (needs the reference checkout; the fixtures themselves are committed). The checkout's
root is the first argument, or the environment variable WT_REFERENCE_ROOT:
    python tests/golden/make_golden.py <reference root>            # solver fixtures
    python tests/golden/make_golden.py <reference root> --frames   # wire frames (frames.npz)
"""
import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, '..', '..', 'oracle'))
from warp_shim import RefKernels  # noqa: E402

Q = 19


def feq(C, W, rho, u):
    """Second-order equilibrium (float64), shape (19, n)."""
    c = np.array(C, np.float64)
    cu = 3.0 * (u @ c.T)                      # (n, 19)
    usq = 1.5 * (u * u).sum(1)
    return (np.array(W)[None, :] * rho[:, None] * (1 + cu + 0.5 * cu * cu - usq[:, None])).T


def random_state(K, dims, rng, real):
    """A far-from-equilibrium state that drives every branch of step_kernel: |u| > 0.35
    (velocity clamp), mac rho outside [0.9, 1.1] (face clamp), negative outlet ux."""
    nx, ny, nz = dims
    n = nx * ny * nz
    rho = rng.uniform(0.85, 1.15, n)
    u = rng.uniform(-0.3, 0.3, (n, 3))
    fs = []
    for _ in range(2):
        f = feq(K.C, K.W, rho, u) + rng.normal(0, 0.004, (Q, n)) * np.array(K.W)[:, None]
        fs.append(np.ascontiguousarray(f.reshape(-1)).astype(real))
    mac = np.empty((n, 4))
    mac[:, :3] = rng.uniform(-0.2, 0.2, (n, 3))
    mac[:, 3] = rng.uniform(0.8, 1.2, n)
    return fs, mac.astype(real)


def random_mask(dims, rng):
    nx, ny, nz = dims
    n = nx * ny * nz
    r = rng.random(n)
    solid = np.zeros(n, np.uint8)
    solid[r < 0.12] = 1
    solid[(r >= 0.12) & (r < 0.17)] = 2
    solid[(r >= 0.17) & (r < 0.18)] = 3          # any non-zero byte is solid; only 1 counts in forces
    return solid


def sphere_mask(dims, c, r, belt):
    nx, ny, nz = dims
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing='ij')
    inside = (x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
    solid = inside.astype(np.uint8).reshape(-1)
    if belt:
        solid.reshape(nz, ny, nx)[:, 0, :] = 2
    return solid


def case_random(K, real, dims, seed, steps_list, name):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    solid = random_mask(dims, rng)
    f, mac = random_state(K, dims, rng, real)
    out = dict(dims=np.array(dims), solid=solid, f0_in=f[0].copy(), f1_in=f[1].copy(), mac_in=mac.copy(),
               uin=real(0.05), tau=real(0.506), smag=real(0.16), steps=np.array(steps_list))
    cur, done = 0, 0
    for k in steps_list:
        while done < k:
            K.step(f[cur], f[1 - cur], solid, mac, nx, ny, nz, 0.05, 0.506, 0.16)
            cur ^= 1
            done += 1
        forces = np.zeros(3, real)
        K.force(f[cur], solid, forces, nx, ny, nz)
        out[f'f_cur_{k}'] = f[cur].copy()
        out[f'f_old_{k}'] = f[1 - cur].copy()
        out[f'mac_{k}'] = mac.copy()
        out[f'forces_{k}'] = forces
    np.savez_compressed(os.path.join(HERE, name), **out)


def case_sphere(K, real, name, steps=100, frames=True):
    """Inlet flow past a sphere on a moving belt, from equilibrium (the reference's reset)."""
    dims = (32, 16, 16)
    nx, ny, nz = dims
    n = nx * ny * nz
    uin, tau, smag = 0.05, 0.506, 0.16
    solid = sphere_mask(dims, (10, 8, 8), 3.5, belt=True)
    f = [np.zeros(Q * n, real) for _ in range(2)]
    mac = np.zeros((n, 4), real)
    for b in f:
        K.init(b, mac, n, uin)
    out = dict(dims=np.array(dims), solid=solid, uin=real(uin), tau=real(tau), smag=real(smag),
               init_f=f[0].copy(), init_mac=mac.copy(), steps=np.array(steps))
    cur = 0
    for s in range(steps):
        K.step(f[cur], f[1 - cur], solid, mac, nx, ny, nz, uin, tau, smag)
        cur ^= 1
        if s + 1 == 50:
            out['f_cur_50'] = f[cur].copy()
    forces = np.zeros(3, real)
    K.force(f[cur], solid, forces, nx, ny, nz)
    out.update(f_cur=f[cur].copy(), f_old=f[1 - cur].copy(), mac=mac.copy(), forces=forces)
    if frames:
        rng = np.random.default_rng(7)
        npart = 400
        pos = np.zeros((npart, 4), real)
        pos[:, 0] = rng.uniform(0.0, nx, npart)          # some start outside the live box
        pos[:, 1] = rng.uniform(0.0, ny, npart)
        pos[:, 2] = rng.uniform(0.0, nz, npart)
        pos[:, 3] = rng.uniform(0, 60, npart).astype(np.int32)
        pos[:5, :3] = [[10, 8, 8], [9.6, 7.6, 8.2], [2.2, 8, 8], [29.5, 8, 8], [16.0, 3.2, 11.7]]
        spd = np.ones(npart, real)
        out['adv_pos_in'] = pos.copy()
        adv = dict(dt=10.0, uin=uin, max_age=50.0, seed=3, sx=2.0, scy=8.0, scz=8.0, shy=5.0, shz=5.0)
        K.advect(pos, spd, mac, solid, nx, ny, nz, adv['dt'], uin, adv['max_age'], adv['seed'], adv['sx'],
                 adv['scy'], adv['scz'], adv['shy'], adv['shz'])
        out['adv_params'] = np.array([adv[k] for k in ('dt', 'uin', 'max_age', 'seed', 'sx', 'scy', 'scz', 'shy', 'shz')])
        out['adv_pos'] = pos.copy()
        out['adv_spd'] = spd.copy()
        q16 = np.zeros(4 * npart, np.uint16)
        q8 = np.zeros(npart, np.uint8)
        K.pack(pos, spd, q16, q8, nx, ny, nz)
        out['pack_q16'], out['pack_q8'] = q16, q8
        slices = []
        for axis in (0, 1, 2):
            w, h = {2: (nx, ny), 1: (nx, nz), 0: (nz, ny)}[axis]
            for field, (vmin, vmax) in enumerate(((0.0, 1.6), (-1.5, 1.0), (0.0, 4.0), (-0.5, 1.5))):
                index = {0: 11, 1: 8, 2: 7}[axis]
                buf = np.zeros(2 * w * h, np.uint8)
                K.slice(mac, solid, buf, nx, ny, nz, axis, index, field, w, h, uin, 8.0, vmin, vmax)
                slices.append(buf)
                out[f'slice_{axis}_{field}'] = buf
                out[f'slice_{axis}_{field}_args'] = np.array([axis, index, field, 8.0, vmin, vmax])
        # surface points on the sphere (and a few stray ones) with outward normals
        nv = 300
        v = rng.normal(size=(nv, 3))
        v /= np.linalg.norm(v, axis=1, keepdims=True)
        verts = (np.array([10, 8, 8]) + 3.5 * v).astype(real)
        norms = v.astype(real)
        verts[:4] = [[0.2, 0.1, 0.3], [31.5, 15.5, 15.2], [10, 8, 8], [5.0, 0.4, 8.0]]
        norms[3] = [0.0, -1.0, 0.0]
        cp = np.zeros(nv, np.int8)
        K.cp(mac, solid, verts, norms, cp, nx, ny, nz, uin)
        out.update(cp_verts=verts, cp_norms=norms, cp=cp)
    np.savez_compressed(os.path.join(HERE, name), **out)


def load_app(ref, K):
    """The reference server module (server/app.py) imported with the stub warp and the
    reference solver module bound to its names; only its pure ``pack`` is used."""
    import importlib.util
    saved = {k: sys.modules.get(k) for k in ('warp', 'lbm')}
    sys.modules['warp'], sys.modules['lbm'] = K.wp, K.mod
    try:
        spec = importlib.util.spec_from_file_location('_ref_app', os.path.join(ref, 'server', 'app.py'))
        app = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(app)
    finally:
        for k, v in saved.items():
            if v is None:
                del sys.modules[k]
            else:
                sys.modules[k] = v
    return app


def frames(ref):
    """Frames written by the reference's own ``pack`` (server/app.py:23-41) for headers and
    parts shaped like the Engine's (server/app.py:179-193): every combination of parts the
    Engine sends, odd part sizes so the 8-byte padding is exercised."""
    K = RefKernels(ref, np.float32)
    app = load_app(ref, K)
    rng = np.random.default_rng(21)
    cases = [  # (numP, slice (w, h) or None, numVerts)
        (13, (12, 7), 5), (2000, None, 0), (0, (33, 9), 0), (0, None, 0), (5, None, 301)]
    out = {}
    for k, (num_p, wh, nv) in enumerate(cases):
        header = {'type': 'frame', 'dims': [64, 28, 36], 'numP': num_p, 'numVerts': nv,
                  'forces': [float(v) for v in rng.normal(size=3) * 1e-2], 'steps': int(rng.integers(1, 40)),
                  'mlups': float(rng.uniform(0, 5e4)), 'running': bool(k % 2 == 0)}
        parts = []
        if num_p:
            parts.append(('parts16', rng.integers(0, 65536, 4 * num_p).astype(np.uint16)))
            parts.append(('parts8', rng.integers(0, 256, num_p).astype(np.uint8)))
        if wh:
            parts.append(('slice', rng.integers(0, 256, 2 * wh[0] * wh[1]).astype(np.uint8)))
            header.update(sliceW=wh[0], sliceH=wh[1], sliceAxis=k % 3)
        if nv:
            parts.append(('cp', rng.integers(-128, 128, nv).astype(np.int8)))
        data = app.pack(header, parts)
        out[f'frame_{k}'] = np.frombuffer(data, np.uint8)
        out[f'header_{k}'] = np.frombuffer(json.dumps(header).encode(), np.uint8)
        out[f'names_{k}'] = np.array([n for n, _ in parts] or [''])
        for name, arr in parts:
            out[f'{name}_{k}'] = arr
    out['cases'] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, 'frames.npz'), **out)


def reference_root(argv):
    """The reference checkout: the first non-option argument, else $WT_REFERENCE_ROOT."""
    args = [a for a in argv[1:] if not a.startswith('--')]
    ref = args[0] if args else os.environ.get('WT_REFERENCE_ROOT')
    if not ref:
        sys.exit('usage: make_golden.py <reference root> [--frames] (or set WT_REFERENCE_ROOT)')
    if not os.path.exists(os.path.join(ref, 'server', 'lbm.py')):
        sys.exit(f'{ref!r} does not hold server/lbm.py of the reference')
    return ref


def main():
    ref = reference_root(sys.argv)
    if '--frames' in sys.argv:
        frames(ref)
        return
    t0 = time.time()
    meta = {}
    for real, tag in ((np.float32, 'f32'), (np.float64, 'f64')):
        K = RefKernels(ref, real)
        meta['gen_source_sha1'] = hashlib.sha1(K.src.encode()).hexdigest()
        case_random(K, real, (12, 8, 10), 11, [1, 3, 8], f'random_12x8x10_{tag}.npz')
        case_random(K, real, (4, 4, 4), 12, [1, 4], f'random_4x4x4_{tag}.npz')
        case_random(K, real, (28, 6, 5), 13, [2], f'random_28x6x5_{tag}.npz')
        case_sphere(K, real, f'sphere_32x16x16_{tag}.npz', frames=(real is np.float32))
        print(tag, 'done', round(time.time() - t0, 1), 's', flush=True)
    with open(os.path.join(HERE, 'SOURCE.txt'), 'w') as fh:
        fh.write('Golden vectors generated by tests/golden/make_golden.py from the reference\n'
                 'RICKxxROLLING/wind-tunnel server/lbm.py run under oracle/warp_shim.py.\n'
                 f'gen_source() sha1: {meta["gen_source_sha1"]}\n'
                 f'numpy {np.__version__}\n')


if __name__ == '__main__':
    main()
