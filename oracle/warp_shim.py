"""Stub-``warp`` shim that executes the reference solver's OWN kernel code on the CPU.

TEST INFRASTRUCTURE ONLY. Nothing in the product imports this module; it exists to
generate golden vectors (``tests/golden/make_golden.py``) from the reference source
``server/lbm.py`` of RICKxxROLLING/wind-tunnel, which needs the reference checkout
on disk and therefore only runs where that checkout is mounted.

How it works
------------
The reference kernels are NVIDIA Warp kernels (``warp-lang==1.17.0``, pinned in
``requirements.txt:1``). Warp is not installed here, so a stand-in ``warp`` module is
placed in ``sys.modules`` before ``server/lbm.py`` is imported:

* ``@wp.kernel`` / ``@wp.func`` are identity decorators; ``wp.tid()`` returns the
  thread index of the current launch; a launch is a serial loop over ``tid``. That is
  the order Warp's CPU backend uses, which fixes the reference's read/write race on
  ``mac`` (face cells read ``mac`` of an interior neighbour that the same launch
  writes, ``server/lbm.py:87`` vs ``:166``): a neighbour with a smaller linear index
  has already been updated, a larger one has not.
* Scalars are ``numpy.float32`` (or ``numpy.float64`` for the fp64 goldens). Python
  float literals in the kernel text combine with them as float32 (numpy's weak scalar
  promotion), which matches Warp's treatment of float literals inside float32 kernels.
  ``float(...)`` inside kernels is rebound to the working precision.
* Builtins follow Warp 1.17's published definitions: ``clamp(x,a,b)=min(max(x,a),b)``,
  ``lerp(a,b,t)=a*(1-t)+b*t``, ``length(v)=sqrt(v.x*v.x+v.y*v.y+v.z*v.z)``,
  ``round`` rounds half away from zero, ``atomic_add`` is a serial add.
* ``wp.rand_init``/``wp.randf`` (Warp's RNG, ``server/lbm.py:256-259``) are not
  reproduced. The shim substitutes the project's own counter-based RNG
  (``oracle_rng_*`` in ``lbm_oracle.cpp``) so that respawn positions are
  deterministic; respawn parity against real Warp is therefore unpinned.

The generated kernels (``gen_source()``, ``server/lbm.py:60-198``) are exec'd from the
reference's own generator output; the hand-written ones (``server/lbm.py:201-368``)
are called directly from the imported module.
"""
import importlib.util
import math
import sys
import types

import numpy as np

_REF_LBM = 'server/lbm.py'

# project RNG (same constants as oracle/lbm_oracle.cpp and the CUDA kernels):
# PCG-RXS-M-XS 32-bit output hash (Jarzynski & Olano, JCGT 2020)
_M32 = 0xFFFFFFFF


def pcg_hash(v):
    state = (v * 747796405 + 2891336453) & _M32
    word = (((state >> ((state >> 28) + 4)) ^ state) * 277803737) & _M32
    return ((word >> 22) ^ word) & _M32


def rng_init(seed, i):
    return pcg_hash((pcg_hash(seed & _M32) + (i & _M32)) & _M32)


def make_stub(real):
    """A stand-in ``warp`` module whose scalar type is ``real`` (np.float32/np.float64)."""
    wp = types.ModuleType('warp')
    wp._tid = 0
    wp.REAL = real

    def tid():
        return wp._tid

    def _deco(f=None, **_kw):
        if f is None:
            return lambda g: g
        return f

    def clamp(x, a, b):
        if isinstance(x, (int, np.integer)) and isinstance(a, (int, np.integer)):
            return min(max(int(x), int(a)), int(b))
        x = real(x)
        lo, hi = real(a), real(b)
        return real(min(max(x, lo), hi))

    def wmax(a, b):
        if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
            return max(a, b)
        a, b = real(a), real(b)
        return b if b > a else a

    def wmin(a, b):
        if isinstance(a, (int, np.integer)) and isinstance(b, (int, np.integer)):
            return min(a, b)
        a, b = real(a), real(b)
        return b if b < a else a

    def vec(*a):
        return np.array([real(v) for v in a], dtype=real)

    def wround(x):
        xd = float(x)
        return real(math.copysign(math.floor(abs(xd) + 0.5), xd))

    def lerp(a, b, t):
        t = real(t)
        return a * (real(1.0) - t) + b * t

    def length(v):
        return real(np.sqrt(real(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])))

    def atomic_add(arr, i, v):
        arr[i] = arr[i] + v

    class _RandState:
        __slots__ = ('s',)

        def __init__(self, s):
            self.s = s

    def rand_init(seed, i):
        return _RandState(rng_init(int(seed), int(i)))

    def randf(st):
        st.s = pcg_hash(st.s)
        return real(np.float32(st.s >> 8) * np.float32(1.0 / 16777216.0))

    wp.tid = tid
    wp.kernel = _deco
    wp.func = _deco
    wp.set_module_options = lambda *a, **k: None
    wp.array = lambda *a, **k: None
    wp.float32 = real
    wp.uint8 = np.uint8
    wp.uint16 = np.uint16
    wp.int8 = np.int8
    wp.vec2 = vec
    wp.vec3 = vec
    wp.vec4 = vec
    wp.clamp = clamp
    wp.max = wmax
    wp.min = wmin
    wp.sqrt = lambda x: real(np.sqrt(real(x)))
    wp.floor = lambda x: real(np.floor(real(x)))
    wp.round = wround
    wp.lerp = lerp
    wp.length = length
    wp.atomic_add = atomic_add
    wp.rand_init = rand_init
    wp.randf = randf
    return wp


class RefKernels:
    """The reference's kernels, runnable serially in tid order at precision ``real``."""

    def __init__(self, ref_root, real=np.float32):
        self.real = real
        self.wp = make_stub(real)
        saved = sys.modules.get('warp')
        sys.modules['warp'] = self.wp
        try:
            name = f'_ref_lbm_{np.dtype(real).name}'
            spec = importlib.util.spec_from_file_location(name, f'{ref_root}/{_REF_LBM}')
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            self.src = mod.gen_source()           # generated with the builtin float
            mod.float = real                      # then kernels see float32 casts
            g = {'__name__': f'_ref_lbm_gen_{np.dtype(real).name}', 'float': real}
            exec(compile(self.src, 'lbm_gen.py', 'exec'), g)
        finally:
            if saved is None:
                del sys.modules['warp']
            else:
                sys.modules['warp'] = saved
        self.mod = mod
        self.gen = g
        self.C, self.W, self.OPP = mod.C, mod.W, mod.OPP
        self.RESOLUTIONS, self.BYTES_PER_CELL, self.CP_RANGE = mod.RESOLUTIONS, mod.BYTES_PER_CELL, mod.CP_RANGE

    def launch(self, kernel, dim, *inputs):
        wp = self.wp
        for t in range(dim):
            wp._tid = t
            kernel(*inputs)

    # ---- the reference's kernels, by name ----
    def init(self, f, mac, n, uin):
        self.launch(self.gen['init_kernel'], n, f, mac, n, self.real(uin))

    def step(self, fin, fout, solid, mac, nx, ny, nz, uin, tau, smag):
        r = self.real
        self.launch(self.gen['step_kernel'], nx * ny * nz, fin, fout, solid, mac, nx, ny, nz, r(uin), r(tau), r(smag))

    def force(self, fcur, solid, forces, nx, ny, nz):
        self.launch(self.gen['force_kernel'], nx * ny * nz, fcur, solid, forces, nx, ny, nz)

    def advect(self, pos, spd, mac, solid, nx, ny, nz, dt, uin, max_age, seed, sx, scy, scz, shy, shz):
        r = self.real
        self.launch(self.mod.advect_kernel, len(pos), pos, spd, mac, solid, nx, ny, nz, r(dt), r(uin), r(max_age),
                    int(seed), r(sx), r(scy), r(scz), r(shy), r(shz))

    def pack(self, pos, spd, q16, q8, nx, ny, nz):
        self.launch(self.mod.pack_particles, len(pos), pos, spd, q16, q8, nx, ny, nz)

    def slice(self, mac, solid, out, nx, ny, nz, axis, index, field, w, h, uin, lref, vmin, vmax):
        r = self.real
        self.launch(self.mod.slice_kernel, w * h, mac, solid, out, nx, ny, nz, axis, index, field, w,
                    r(uin), r(lref), r(vmin), r(vmax))

    def cp(self, mac, solid, verts, norms, out, nx, ny, nz, uin):
        r = self.real
        self.launch(self.mod.cp_kernel, len(verts), mac, solid, verts, norms, out, nx, ny, nz, r(uin),
                    r(self.CP_RANGE))
