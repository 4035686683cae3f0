"""ctypes wrapper around ``liblbm_oracle.so`` -- TEST INFRASTRUCTURE ONLY.

The oracle is the parity checker for the CUDA kernels and the timed CPU baseline. Only
``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs may use it. It is a
CPU restatement of ``server/lbm.py`` (RICKxxROLLING/wind-tunnel); see lbm_oracle.cpp for
the per-kernel citations. Buffers are numpy arrays in the reference's layout: populations
SoA ``f[i * n + idx]`` with ``idx = x + nx * (y + ny * z)``, ``mac`` as (n, 4) rows
``(ux, uy, uz, rho)``, ``solid`` u8 (0 fluid, 1 solid, 2 moving belt).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'liblbm_oracle.so')

F32, F16, BF16, F64 = 0, 1, 2, 3
CP_RANGE = 1.2
Q = 19
CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1])
CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1])
W = np.array([1 / 3 if i == 0 else (1 / 18 if abs(CX[i]) + abs(CY[i]) + abs(CZ[i]) == 1 else 1 / 36)
              for i in range(Q)])

_lib = None


def build():
    subprocess.run(['make', '-s', '-C', HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        vp, i32, i64, f32, f64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_float, ctypes.c_double
        L.oracle_num_threads.argtypes = [i32]
        L.oracle_init.argtypes = [i32, vp, vp, i64, f64]
        L.oracle_step.argtypes = [i32, vp, vp, vp, vp, i32, i32, i32, f64, f64, f64, i32, i32]
        L.oracle_force.argtypes = [i32, vp, vp, i32, i32, i32, vp, vp, vp]
        L.oracle_mass.argtypes = [i32, vp, vp, i64, vp]
        L.oracle_advect_f32.argtypes = [vp, vp, vp, vp, i32, i32, i32, i64, f32, f32, f32, i32, f32, f32, f32, f32, f32]
        L.oracle_pack_f32.argtypes = [vp, vp, vp, vp, i32, i32, i32, i64]
        L.oracle_slice_f32.argtypes = [vp, vp, vp, i32, i32, i32, i32, i32, i32, i32, i32, f32, f32, f32, f32]
        L.oracle_cp_f32.argtypes = [vp, vp, vp, vp, vp, i32, i32, i32, i64, f32, f32]
        L.oracle_rng_hash.argtypes = [ctypes.c_uint32]
        L.oracle_rng_hash.restype = ctypes.c_uint32
        L.oracle_set_shift.argtypes = [f64]
        L.oracle_set_shift.restype = None
        _lib = L
    return _lib


def _p(a):
    assert a.flags['C_CONTIGUOUS']
    return a.ctypes.data_as(ctypes.c_void_p)


def store_dtype(prec):
    # numpy has no bfloat16: bf16 populations are carried as raw uint16 bit patterns
    return {F32: np.float32, F16: np.float16, BF16: np.uint16, F64: np.float64}[prec]


def real_dtype(prec):
    return np.float64 if prec == F64 else np.float32


def set_threads(n):
    return lib().oracle_num_threads(int(n))


def _chk(rc, what):
    if rc != 0:
        raise RuntimeError(f'oracle {what} failed: {rc}')


def shift_values(U):
    """float32 shifts e_i of half-width storage: w_i (1 + 3 c_xi U + 4.5 c_xi^2 U^2 - 1.5 U^2)
    in double, rounded once (oracle_set_shift); U = 0 gives the rest weights."""
    if U == 0.0:
        return W.astype(np.float32)
    cx = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0], np.float64)
    out = []
    for i in range(Q):
        cu = 3.0 * cx[i] * U
        out.append(W[i] * (1.0 + cu + 0.5 * cu * cu - 1.5 * U * U))
    return np.array(out, np.float32)


class Lattice:
    """The reference Solver's device state held in host numpy arrays (server/lbm.py:398-413)."""

    def __init__(self, dims, prec=F32, collision=0, shift_u=0.0):
        self.collision = int(collision)  # 0 reference order, 1 moment-space form
        # fp16/bf16 storage shift velocity (the library's wt_grid.shift_u; 0 = rest weights)
        self.shift_u = float(shift_u)
        self.nx, self.ny, self.nz = (int(d) for d in dims)
        self.n = n = self.nx * self.ny * self.nz
        self.prec = prec
        sd, rd = store_dtype(prec), real_dtype(prec)
        self.f = [np.zeros(Q * n, sd) for _ in range(2)]
        self.solid = np.zeros(n, np.uint8)
        self.mac = np.zeros((n, 4), rd)
        self.cur = 0

    def _shift(self):
        lib().oracle_set_shift(self.shift_u)

    def reset(self, uin):
        self._shift()
        for buf in self.f:
            _chk(lib().oracle_init(self.prec, _p(buf), _p(self.mac), self.n, float(uin)), 'init')

    def step(self, steps, uin, tau, smag, serial=False):
        L = lib()
        self._shift()
        for _ in range(int(steps)):
            _chk(L.oracle_step(self.prec, _p(self.f[self.cur]), _p(self.f[1 - self.cur]), _p(self.solid),
                               _p(self.mac), self.nx, self.ny, self.nz, float(uin), float(tau), float(smag),
                               1 if serial else 0, self.collision), 'step')
            self.cur ^= 1

    def forces(self):
        """(reference-order float sums, fp64 sums, fp64 sums without floor links)."""
        rd = real_dtype(self.prec)
        ref = np.zeros(3, rd)
        d = np.zeros(3, np.float64)
        b = np.zeros(3, np.float64)
        self._shift()
        _chk(lib().oracle_force(self.prec, _p(self.f[self.cur]), _p(self.solid), self.nx, self.ny, self.nz,
                                _p(ref), _p(d), _p(b)), 'force')
        return ref, d, b

    def mass(self):
        out = np.zeros(1, np.float64)
        self._shift()
        _chk(lib().oracle_mass(self.prec, _p(self.f[self.cur]), _p(self.solid), self.n, _p(out)), 'mass')
        return float(out[0])

    def populations(self, which=None):
        """Populations of buffer ``which`` (default: current) as float64, unshifted, shape (19, n)."""
        buf = self.f[self.cur if which is None else which]
        e = shift_values(self.shift_u).astype(np.float64)[:, None]
        if self.prec == F16:
            v = buf.astype(np.float64).reshape(Q, self.n) + e
        elif self.prec == BF16:
            v = (buf.astype(np.uint32) << 16).view(np.float32).astype(np.float64).reshape(Q, self.n) + e
        else:
            v = buf.astype(np.float64).reshape(Q, self.n)
        return v


def advect(pos, spd, mac, solid, dims, dt, uin, max_age, seed, sx, scy, scz, shy, shz):
    nx, ny, nz = dims
    _chk(lib().oracle_advect_f32(_p(pos), _p(spd), _p(mac), _p(solid), nx, ny, nz, len(spd), dt, uin, max_age,
                                 int(seed), sx, scy, scz, shy, shz), 'advect')


def pack(pos, spd, dims):
    nx, ny, nz = dims
    q16 = np.zeros(4 * len(spd), np.uint16)
    q8 = np.zeros(len(spd), np.uint8)
    _chk(lib().oracle_pack_f32(_p(pos), _p(spd), _p(q16), _p(q8), nx, ny, nz, len(spd)), 'pack')
    return q16, q8


def slice_dims(dims, axis):
    nx, ny, nz = dims
    return {2: (nx, ny), 1: (nx, nz), 0: (nz, ny)}[axis]


def slice_(mac, solid, dims, axis, index, field, uin, lref, vmin, vmax):
    nx, ny, nz = dims
    w, h = slice_dims(dims, axis)
    out = np.zeros(2 * w * h, np.uint8)
    _chk(lib().oracle_slice_f32(_p(mac), _p(solid), _p(out), nx, ny, nz, axis, index, field, w, h, uin, lref,
                                vmin, vmax), 'slice')
    return out


def cp(mac, solid, verts, norms, dims, uin):
    nx, ny, nz = dims
    out = np.zeros(len(verts), np.int8)
    _chk(lib().oracle_cp_f32(_p(mac), _p(solid), _p(verts), _p(norms), _p(out), nx, ny, nz, len(verts), uin,
                             CP_RANGE), 'cp')
    return out
