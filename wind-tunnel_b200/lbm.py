"""B200 lattice-Boltzmann wind tunnel (D3Q19, regularized collision + Smagorinsky LES).

Drop-in replacement for the reference's ``server/lbm.py`` (RICKxxROLLING/wind-tunnel):
the same module exports (``RESOLUTIONS``, ``BYTES_PER_CELL``, ``Solver``) and the same
``Solver`` methods and attributes that ``server/app.py`` drives
(``server/lbm.py:398-482``). The work runs in hand-written sm_100a kernels in
``libwt.so`` called through the C ABI of ``include/wt.h``; torch tensors serve only as
device buffers. There is no CPU path: constructing a Solver without a CUDA device raises.

Lattice frame as in the reference: x streamwise (flow +x), y vertical, z span; cell
centres at integer coordinates; cell index ``idx = x + nx * (y + ny * z)``.
"""
import ctypes

import numpy as np
import torch

import wire
import wtlib as W
from wtlib import call, ptr

Q = 19

# grid presets (server/lbm.py:21-29)
RESOLUTIONS = {
    'test': (64, 28, 36),
    'low': (128, 56, 72),
    'medium': (176, 80, 96),
    'high': (256, 112, 136),
    'ultra': (352, 144, 176),
    'extreme': (448, 192, 224),
    'max': (544, 224, 272),
}

CP_RANGE = 1.2  # server/lbm.py:395

_POP_BYTES = {W.F32: 4, W.F16: 2, W.F64: 8, W.BF16: 2}
_TORCH_POP = {W.F32: torch.float32, W.F16: torch.float16, W.BF16: torch.bfloat16, W.F64: torch.float64}


def bytes_per_cell(precision='fp32'):
    """Device bytes per cell: two population buffers, two mac buffers, solid and code bytes."""
    prec = W.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    mac = 32 if prec == W.F64 else 16
    return 2 * Q * _POP_BYTES[prec] + 2 * mac + 2


# The reference's name for the admission footprint (server/lbm.py:30, used by app.py:76).
BYTES_PER_CELL = bytes_per_cell('fp32')


def estimate_bytes(dims, precision='fp32', particles=0, num_verts=0):
    """Device bytes of a Solver before it exists: the per-cell state, particle buffers
    (pos 16 + speed 4 + packed 9 bytes each, twice the packed bytes for the frame buffer),
    the slice buffer and the force partials. The link list (8 bytes per fluid cell next to a
    wall) is not included; Solver.device_bytes() gives the exact figure afterwards."""
    nx, ny, nz = (int(d) for d in dims)
    slice_max = max(nx * ny, nx * nz, nz * ny)
    return (bytes_per_cell(precision) * nx * ny * nz + particles * (20 + 2 * 9) + 2 * 2 * slice_max
            + num_verts * 26 + 8 * int(W.lib().wt_reduce_scratch_len(0)) + 4096)


def state_layout(dims, precision='fp32'):
    """Byte offsets of a Solver's per-cell state in one block of device memory (the two
    population buffers, the two mac buffers, solid and code, each 256-byte aligned), and the
    block's size: {'f0': (offset, bytes), ...}, total."""
    prec = W.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
    nx, ny, nz = (int(d) for d in dims)
    n = nx * ny * nz
    mac = 32 if prec == W.F64 else 16
    parts = [('f0', Q * n * _POP_BYTES[prec]), ('f1', Q * n * _POP_BYTES[prec]), ('mac0', n * mac), ('mac1', n * mac),
             ('solid', n), ('code', n)]
    out, off = {}, 0
    for name, nbytes in parts:
        out[name] = (off, nbytes)
        off += (nbytes + 255) // 256 * 256
    return out, off


def _device(device):
    if not torch.cuda.is_available():
        raise RuntimeError('wind-tunnel_b200 needs a CUDA device; there is no CPU path')
    if device is None:
        return torch.device('cuda', torch.cuda.current_device())
    if isinstance(device, int):
        return torch.device('cuda', device)
    d = torch.device(device)
    if d.type != 'cuda':
        raise RuntimeError(f'device {device!r} is not a CUDA device; there is no CPU path')
    return d if d.index is not None else torch.device('cuda', torch.cuda.current_device())


class Solver:
    """One tunnel. Method-for-method the reference Solver (server/lbm.py:398-482).

    Extra keyword arguments: ``precision`` ('fp32' as the reference, 'fp16'/'bf16' for
    shifted half-width population storage, 'fp64' for the oracle run), ``collision``
    ('exact' reference operation order or 'fast' moment-space form; by default exact for
    fp32/fp64 and fast for fp16/bf16), ``stream`` (a ``torch.cuda.Stream``; by default each
    Solver owns one) and ``seed`` (particle initialisation; the reference draws from an
    unseeded generator).
    """

    def __init__(self, dims, device=None, precision='fp32', stream=None, seed=None, collision=None,
                 shift='free-stream', storage=None):
        self.dev = _device(device)
        self.nx, self.ny, self.nz = (int(d) for d in dims)
        self.n = n = self.nx * self.ny * self.nz
        call('wt_check_dims', self.nx, self.ny, self.nz)
        self.precision = W.PRECISIONS[precision] if isinstance(precision, str) else int(precision)
        if self.precision not in _TORCH_POP:
            raise ValueError(f'unknown precision {precision!r}')
        # 'exact': the reference's expressions in its order (default for fp32/fp64, the
        # drop-in form); 'fast': the moment-space form (default for fp16/bf16 storage)
        if collision is None:
            collision = 'fast' if self.precision in (W.F16, W.BF16) else 'exact'
        if collision not in ('exact', 'fast'):
            raise ValueError(f'unknown collision form {collision!r}')
        self.collision = collision
        if shift not in ('free-stream', 'rest'):
            raise ValueError(f'unknown storage shift {shift!r}')
        self.shift_mode = shift
        self.stream = stream if stream is not None else torch.cuda.Stream(self.dev)
        mac_dt = torch.float64 if self.precision == W.F64 else torch.float32
        with torch.cuda.device(self.dev), torch.cuda.stream(self.stream):
            # zero-filled like the reference's wp.zeros buffers (server/lbm.py:404-407)
            if storage is None:
                self.f = [torch.zeros(Q * n, dtype=_TORCH_POP[self.precision], device=self.dev) for _ in range(2)]
                self.mac = [torch.zeros((n, 4), dtype=mac_dt, device=self.dev) for _ in range(2)]
                self.solid = torch.zeros(n, dtype=torch.uint8, device=self.dev)
                self.code = torch.zeros(n, dtype=torch.uint8, device=self.dev)
            else:
                # the per-cell state in a caller's block of device memory (uint8, 256-byte aligned,
                # state_layout's size at least), e.g. a range of a serving arena
                layout, total = state_layout(dims, self.precision)
                if storage.dtype != torch.uint8 or storage.dim() != 1 or storage.numel() < total:
                    raise ValueError(f'storage must be a 1-D uint8 tensor of at least {total} bytes')
                if storage.device != self.dev or storage.data_ptr() % 256:
                    raise ValueError('storage must be 256-byte aligned memory on the Solver\'s device')
                part = {k: storage[o:o + nb] for k, (o, nb) in layout.items()}
                self.f = [part[k].view(_TORCH_POP[self.precision]) for k in ('f0', 'f1')]
                self.mac = [part[k].view(mac_dt).view(n, 4) for k in ('mac0', 'mac1')]
                self.solid, self.code = part['solid'], part['code']
                for t in (*self.f, *self.mac, self.solid, self.code):
                    t.zero_()
            self.forces_dev = torch.zeros(6, dtype=torch.float64, device=self.dev)
            self.mass_dev = torch.zeros(1, dtype=torch.float64, device=self.dev)
            self.status_dev = torch.zeros(1, dtype=torch.int32, device=self.dev)
            self.partials = torch.empty(int(W.lib().wt_reduce_scratch_len(0)), dtype=torch.float64, device=self.dev)
            self.slice_max = max(self.nx * self.ny, self.nx * self.nz, self.nz * self.ny)
            self.slice_buf = torch.zeros(self.slice_max * 2, dtype=torch.uint8, device=self.dev)
            self.link_cells = torch.zeros(0, dtype=torch.int32, device=self.dev)
            self.link_masks = torch.zeros(0, dtype=torch.int32, device=self.dev)
        self.n_links = 0
        self.grid = W.Grid(self.nx, self.ny, self.nz, self.precision,
                           (ctypes.c_void_p * 2)(self.f[0].data_ptr(), self.f[1].data_ptr()),
                           (ctypes.c_void_p * 2)(self.mac[0].data_ptr(), self.mac[1].data_ptr()),
                           self.solid.data_ptr(), self.code.data_ptr(), 0,
                           W.COLLIDE_FAST if collision == 'fast' else W.COLLIDE_EXACT)
        self.grid.status = self.status_dev.data_ptr()
        self.gp = ctypes.byref(self.grid)
        self.sh = W.stream_handle(self.stream)
        self.cur = 0
        self.num_p = 0
        self.num_verts = 0
        self.seed = 1
        self.rng = np.random.default_rng(seed)
        self._host = {}
        self._pending = None
        self.stream.synchronize()

    def recycle(self, seed=None):
        """Return to the state right after construction with ``seed``, keeping the device and
        pinned buffers: a new tunnel of the same grid, precision and collision form (a serving
        session replacing one that left) then needs no allocation, which would hold driver and
        interpreter locks while other tunnels are being launched. Populations, macros, mask and
        codes are zeroed, and links, particles, surface, tile and pending frames are dropped,
        as a new Solver has them."""
        self.synchronize()
        with torch.cuda.stream(self.stream):
            for t in (*self.f, *self.mac, self.solid, self.code, self.status_dev):
                t.zero_()
        self.n_links = 0
        self.grid.tile = 0
        self.grid.shift_u = 0.0
        self.cur = 0
        self.num_p = 0
        self.num_verts = 0
        self.seed = 1
        self.rng = np.random.default_rng(seed)
        self._pending = None
        self._pk_pending = None
        self._pk_layout_key = None  # the next layout zeroes the packed-frame buffer
        self.stream.synchronize()

    def set_tile(self, tile):
        """Select a step-kernel tile variant (see wtlib.step_tiles; 0 = library default)."""
        self.grid.tile = int(tile)

    @property
    def tile(self):
        return int(self.grid.tile)

    # ---- set-up (server/lbm.py:415-440) ----
    def reset(self, uin):
        """Equilibrium at rho = 1, u = (uin, 0, 0) in both population buffers (init_kernel).
        fp16/bf16 storage is shifted by the equilibrium at u = (uin, 0, 0) from here on
        (``shift_u``; 0 keeps the rest weights, e.g. for comparisons with that form)."""
        if self.precision in (W.F16, W.BF16) and self.shift_mode == 'free-stream':
            self.grid.shift_u = float(uin)
        else:
            self.grid.shift_u = 0.0
        for b in range(2):
            call('wt_init_eq', self.precision, ptr(self.f[b]), ptr(self.mac[b]), self.n, float(uin),
                 float(self.grid.shift_u), self.sh)

    def set_solid(self, arr):
        """Upload the voxel mask (0 fluid, 1 solid, 2 moving belt) and rebuild the per-cell
        codes and the compacted momentum-exchange link list."""
        arr = np.asarray(arr)
        assert arr.size == self.n
        # no copy of a mask that is already contiguous uint8, no second staging of pinned memory
        a = np.ascontiguousarray(arr.reshape(-1), dtype=np.uint8)
        host = torch.from_numpy(a if a.flags.writeable else a.copy())  # uploads are read-only views
        with torch.cuda.stream(self.stream):
            self.solid.copy_(host if host.is_pinned() else host.pin_memory(), non_blocking=True)
            call('wt_build_codes', self.gp, self.sh)
            scratch = torch.empty(int(W.lib().wt_links_scratch_len(self.n)), dtype=torch.int64, device=self.dev)
            count = torch.zeros(1, dtype=torch.int64, device=self.dev)
            call('wt_links_scan', self.gp, ptr(scratch), ptr(count), self.sh)
            self.n_links = int(count.to('cpu', non_blocking=False).item())
            cap = max(1, self.n_links)
            self.link_cells = torch.empty(cap, dtype=torch.int32, device=self.dev)
            self.link_masks = torch.empty(cap, dtype=torch.int32, device=self.dev)
            call('wt_links_fill', self.gp, ptr(scratch), ptr(self.link_cells), ptr(self.link_masks), cap, self.sh)
        self.stream.synchronize()

    def set_surface(self, verts, norms):
        # writable copies where needed: uploads arrive as read-only views of the message bytes
        verts = np.require(np.asarray(verts, np.float32).reshape(-1, 3), requirements=['C', 'W'])
        norms = np.require(np.asarray(norms, np.float32).reshape(-1, 3), requirements=['C', 'W'])
        self.num_verts = len(verts)
        with torch.cuda.stream(self.stream):
            self.verts = torch.from_numpy(verts).to(self.dev, non_blocking=False)
            self.norms = torch.from_numpy(norms).to(self.dev, non_blocking=False)
            self.cp_buf = torch.zeros(max(1, self.num_verts), dtype=torch.int8, device=self.dev)

    def set_particles(self, count, p):
        """Streamline particles in the rake box (server/lbm.py:429-440), from this Solver's
        seeded generator."""
        rng = self.rng
        d = np.zeros((count, 4), np.float32)
        d[:, 0] = 2 + rng.random(count) * (self.nx - 8)
        d[:, 1] = p['seedCy'] + (rng.random(count) * 2 - 1) * p['seedHy']
        d[:, 2] = p['seedCz'] + (rng.random(count) * 2 - 1) * p['seedHz']
        d[:, 3] = rng.random(count) * p['maxAge'] * 0.5
        self.num_p = count
        with torch.cuda.stream(self.stream):
            self.pos = torch.from_numpy(d).to(self.dev)
            self.spd = torch.ones(count, dtype=torch.float32, device=self.dev)
            self.q16 = torch.zeros(count * 4, dtype=torch.int16, device=self.dev)
            self.q8 = torch.zeros(count, dtype=torch.uint8, device=self.dev)
        self.stream.synchronize()

    # ---- hot path (server/lbm.py:442-453) ----
    def step(self, steps, p):
        steps = int(steps)
        if steps > 0:
            call('wt_step', self.gp, self.cur, steps, float(p['uIn']), float(p['tau']), float(p['smag']),
                 W.STEP_MAC_ALL_LAST, self.sh)
            self.cur ^= steps & 1
        self.advance_particles(steps, p)

    def advance_particles(self, steps, p):
        """The particle half of step(): one RK2 advection over dt = steps with a fresh seed.
        A tunnel stepped inside a TunnelBatch calls this after the batch's steps."""
        if self.num_p and steps:
            self.seed += 1
            self._advect(float(steps), p)

    def wait_event(self, event):
        """Make this Solver's stream wait for a CUDA event (e.g. a TunnelBatch's steps)."""
        self.stream.wait_event(event)

    def _advect(self, dt, p):
        self._require_float_mac('particles')
        call('wt_advect', ptr(self.pos), ptr(self.spd), ptr(self.mac[self.cur]), ptr(self.solid), self.nx, self.ny,
             self.nz, self.num_p, dt, float(p['uIn']), float(p['maxAge']), self.seed & 0xFFFFFFFF,
             float(p['seedX']), float(p['seedCy']), float(p['seedCz']), float(p['seedHy']), float(p['seedHz']),
             self.sh)

    def slice_dims(self, axis):
        return {2: (self.nx, self.ny), 1: (self.nx, self.nz), 0: (self.nz, self.ny)}[axis]

    # ---- frame outputs (server/lbm.py:458-482) ----
    def _pinned(self, key, shape, dtype):
        t = self._host.get(key)
        if t is None or t.shape != torch.Size(shape) or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, pin_memory=True)
            self._host[key] = t
        return t

    def _require_float_mac(self, what):
        if self.precision == W.F64:
            raise NotImplementedError(f'{what} output needs float mac; the fp64 run reports forces and mass only')

    def launch_frame(self, p, want_cp, copy=True):
        """Queue every frame kernel and (with copy) its device-to-host copy on the Solver's
        stream without waiting; collect_frame() waits once and returns the reference's dict."""
        out = {}
        copies = []
        mac = self.mac[self.cur]
        if self.num_p:
            self._require_float_mac('particles')
            call('wt_pack_particles', ptr(self.pos), ptr(self.spd), ptr(self.q16), ptr(self.q8), self.nx, self.ny,
                 self.nz, self.num_p, self.sh)
            copies.append(('parts16', self.q16, self._pinned('q16', (self.num_p * 4,), torch.int16)))
            copies.append(('parts8', self.q8, self._pinned('q8', (self.num_p,), torch.uint8)))
        sl = p.get('slice')
        if sl and sl.get('field', -1) >= 0:
            self._require_float_mac('slice')
            axis = int(sl['axis'])
            w, h = self.slice_dims(axis)
            dim = (self.nx, self.ny, self.nz)[axis]
            index = max(0, min(dim - 1, int(sl['index'])))
            call('wt_slice', ptr(mac), ptr(self.solid), ptr(self.slice_buf), self.nx, self.ny, self.nz, axis, index,
                 int(sl['field']), float(p['uIn']), float(p['lref']), float(sl['vmin']), float(sl['vmax']), self.sh)
            copies.append(('slice', self.slice_buf[:w * h * 2], self._pinned('slice', (w * h * 2,), torch.uint8)))
            out['sliceW'], out['sliceH'], out['sliceAxis'] = w, h, axis
        if want_cp and self.num_verts:
            self._require_float_mac('surface pressure')
            call('wt_cp', ptr(mac), ptr(self.solid), ptr(self.verts), ptr(self.norms), ptr(self.cp_buf), self.nx,
                 self.ny, self.nz, self.num_verts, float(p['uIn']), CP_RANGE, self.sh)
            copies.append(('cp', self.cp_buf[:self.num_verts], self._pinned('cp', (self.num_verts,), torch.int8)))
        call('wt_forces', self.gp, self.cur, ptr(self.link_cells), ptr(self.link_masks), self.n_links,
             ptr(self.partials), ptr(self.forces_dev), self.sh)
        copies.append(('forces6', self.forces_dev, self._pinned('forces6', (6,), torch.float64)))
        if not copy:
            self._pending = None
            return
        with torch.cuda.stream(self.stream):
            for _, src, dst in copies:
                dst.copy_(src, non_blocking=True)
        self._pending = (out, copies)

    def collect_frame(self):
        out, copies = self._pending
        self._pending = None
        self.stream.synchronize()
        views = {'parts16': np.uint16, 'parts8': np.uint8, 'slice': np.uint8, 'cp': np.int8}
        for key, _, dst in copies:
            a = dst.numpy()
            if key == 'forces6':
                self.last_forces6 = a.copy()
                out['forces'] = [float(v) for v in a[:3]]
            else:
                out[key] = a.view(views[key]).copy()
        return out

    def frame(self, p, want_cp):
        """Reference Solver.frame: particles, slice, surface Cp and forces in one dict."""
        self.launch_frame(p, want_cp)
        return self.collect_frame()

    def _frame_buffers(self, layout, wh):
        # grow-only: frames with and without surface pressure alternate layouts, and pinned
        # allocation is slow. A new layout zeroes the device buffer, so the padding between
        # parts is zero, as pack() writes it.
        key = (self.num_p, wh, layout.total_bytes, tuple(sorted(layout.offsets.items())))
        if getattr(self, '_pk_layout_key', None) == key:
            return
        need = layout.total_bytes
        if getattr(self, '_pk_cap', 0) < need:
            with torch.cuda.stream(self.stream):
                self._pk_dev = torch.zeros(need, dtype=torch.uint8, device=self.dev)
            self._pk_host = torch.empty(need, dtype=torch.uint8, pin_memory=True)
            self._pk_cap = need
        else:
            with torch.cuda.stream(self.stream):
                self._pk_dev.zero_()
        self._pk_layout_key = key

    def _frame_layout(self, p, want_cp):
        sl = p.get('slice')
        slice_on = bool(sl) and sl.get('field', -1) >= 0
        cp_on = bool(want_cp) and self.num_verts > 0
        wh = self.slice_dims(int(sl['axis'])) if slice_on else None
        return wire.FrameLayout(self.num_p, wh, self.num_verts if cp_on else 0), wh, slice_on, cp_on

    def prepare_frame(self, p, want_cp=False):
        """Allocate the device and pinned host buffers of launch_frame_packed ahead of the
        first frame (pinned host allocation is slow)."""
        layout, wh, _, _ = self._frame_layout(p, want_cp)
        self._frame_buffers(layout, wh)

    def launch_frame_packed(self, p, want_cp):
        """The frame kernels of launch_frame, writing straight into one device buffer laid out
        as the wire payload (wire.FrameLayout), the six force components in its 48-byte tail,
        then one device-to-host copy into pinned memory. Nothing waits; collect_frame_packed()
        returns the frame bytes the reference's pack() would send (server/app.py:179-193)."""
        layout, wh, slice_on, cp_on = self._frame_layout(p, want_cp)
        self._frame_buffers(layout, wh)
        sl = p.get('slice')
        base = self._pk_dev.data_ptr()
        mac = self.mac[self.cur]
        extra = {}
        if self.num_p:
            self._require_float_mac('particles')
            call('wt_pack_particles', ptr(self.pos), ptr(self.spd), base + layout.offsets['parts16'],
                 base + layout.offsets['parts8'], self.nx, self.ny, self.nz, self.num_p, self.sh)
        if slice_on:
            self._require_float_mac('slice')
            axis = int(sl['axis'])
            dim = (self.nx, self.ny, self.nz)[axis]
            index = max(0, min(dim - 1, int(sl['index'])))
            call('wt_slice', ptr(mac), ptr(self.solid), base + layout.offsets['slice'], self.nx, self.ny, self.nz,
                 axis, index, int(sl['field']), float(p['uIn']), float(p['lref']), float(sl['vmin']),
                 float(sl['vmax']), self.sh)
            extra = {'sliceW': wh[0], 'sliceH': wh[1], 'sliceAxis': axis}
        if cp_on:
            self._require_float_mac('surface pressure')
            call('wt_cp', ptr(mac), ptr(self.solid), ptr(self.verts), ptr(self.norms), base + layout.offsets['cp'],
                 self.nx, self.ny, self.nz, self.num_verts, float(p['uIn']), CP_RANGE, self.sh)
        call('wt_forces', self.gp, self.cur, ptr(self.link_cells), ptr(self.link_masks), self.n_links,
             ptr(self.partials), base + layout.forces_offset, self.sh)
        with torch.cuda.stream(self.stream):
            tb = layout.total_bytes
            self._pk_host[:tb].copy_(self._pk_dev[:tb], non_blocking=True)
            self._pk_event = torch.cuda.Event()
            self._pk_event.record(self.stream)
        self._pk_pending = (layout, extra)

    def frame_ready(self):
        """True once launch_frame_packed's copy has landed (collect_frame_packed will not wait)."""
        return self._pk_pending is None or self._pk_event.query()

    def collect_frame_packed(self, header):
        """Wait for launch_frame_packed's copy and return the frame bytes. ``header`` holds
        the Engine's keys in its order (type, dims, numP, numVerts, forces, steps, mlups,
        running); forces and the slice keys are filled in here."""
        layout, extra = self._pk_pending
        self._pk_pending = None
        self._pk_event.synchronize()
        host = self._pk_host.numpy()
        f6 = host[layout.forces_offset:layout.forces_offset + 48].view(np.float64)
        self.last_forces6 = f6.copy()
        h = dict(header)
        h['forces'] = [float(v) for v in f6[:3]]
        h.update(extra)
        return layout.frame(h, host)

    # ---- extras used by tests, the serving loop and the benchmark ----
    def forces6(self):
        """[Fx, Fy, Fz] over all solid==1 links, then without links into the y = 0 plane (fp64)."""
        call('wt_forces', self.gp, self.cur, ptr(self.link_cells), ptr(self.link_masks), self.n_links,
             ptr(self.partials), ptr(self.forces_dev), self.sh)
        self.stream.synchronize()
        return self.forces_dev.cpu().numpy().copy()

    def mass(self):
        call('wt_mass', self.gp, self.cur, ptr(self.partials), ptr(self.mass_dev), self.sh)
        self.stream.synchronize()
        return float(self.mass_dev.cpu()[0])

    def populations(self, which=None):
        """Populations of buffer ``which`` (default current) as float64 numpy (19, n),
        with the w_i shift of fp16/bf16 storage removed."""
        self.stream.synchronize()
        f = self.f[self.cur if which is None else which].double().cpu().numpy().reshape(Q, self.n)
        if self.precision in (W.F16, W.BF16):
            f = f + shift_values(float(self.grid.shift_u)).astype(np.float64)[:, None]
        return f

    def macro(self):
        """mac of the current buffer as float64 numpy (n, 4): ux, uy, uz, rho."""
        self.stream.synchronize()
        return self.mac[self.cur].double().cpu().numpy()

    def synchronize(self):
        self.stream.synchronize()

    def device_bytes(self):
        """Bytes of device memory this Solver holds (its tensors; the caching allocator's
        rounding and the frame buffer's reuse come on top)."""
        ts = [*self.f, *self.mac, self.solid, self.code, self.forces_dev, self.mass_dev, self.status_dev,
              self.partials, self.slice_buf, self.link_cells, self.link_masks]
        for k in ('pos', 'spd', 'q16', 'q8', 'verts', 'norms', 'cp_buf', '_pk_dev'):
            t = getattr(self, k, None)
            if t is not None:
                ts.append(t)
        return sum(t.numel() * t.element_size() for t in ts)

    def status(self, clear=True):
        """Device status word: 0, or wtlib.WT_ERR_TIMEOUT if a kernel's bounded wait gave up
        (the populations are then invalid until the next reset)."""
        self.stream.synchronize()
        v = int(self.status_dev.cpu()[0])
        if clear and v:
            self.status_dev.zero_()
            torch.cuda.synchronize(self.dev)
        return v


def shift_values(U):
    """float32 e_i of shifted storage: w_i (1 + 3 c_xi U + 4.5 c_xi^2 U^2 - 1.5 U^2) evaluated
    in double and rounded once (the library's ShiftTables); U = 0 gives w_i."""
    w = _weights()
    cxs = [0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0]
    if U == 0.0:
        return np.array(w, np.float32)
    out = []
    for i in range(Q):
        cu = 3.0 * cxs[i] * U
        out.append(w[i] * (1.0 + cu + 0.5 * cu * cu - 1.5 * U * U))
    return np.array(out, np.float32)


def _weights():
    c = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
         (1, 1, 0), (-1, -1, 0), (1, -1, 0), (-1, 1, 0), (1, 0, 1), (-1, 0, -1), (1, 0, -1), (-1, 0, 1),
         (0, 1, 1), (0, -1, -1), (0, 1, -1), (0, -1, 1)]
    return [1 / 3 if i == 0 else (1 / 18 if sum(map(abs, v)) == 1 else 1 / 36) for i, v in enumerate(c)]
