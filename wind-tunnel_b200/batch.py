"""Many tunnels advanced together (wt_batch_* of include/wt.h).

``TunnelBatch`` groups Solvers of one device, precision and collision form, in one of two
executors:

* ``mode='persistent'``: each step runs one bulk kernel over every tunnel, then one kernel over
  all tunnels' face cells; ``capture(k)`` records k (even) steps as a CUDA graph that
  ``replay()`` launches with a single call. The tile picks the kernel's form: a persistent
  loop over a device work list (tiles 1-5, 7, 18), one block per work-list tile (100 + k), or
  the tunnels' descriptors in the kernel parameters (200 + k, no device work list; these also
  step tunnels by different counts).
* ``mode='streams'``: each tunnel is stepped by the single-tunnel kernel on its own stream, all
  streams running at once after the batch stream's prior work, and the batch stream joins them;
  ``capture(k)`` records that fork and join (k even) as one CUDA graph.
  Each kernel keeps its tunnel's scalars in its constant-bank parameters, so it runs the
  64-register two-cell tile; concurrent tunnels fill each other's tails. On config 4 (24
  tunnels of 0.5-8M cells) it runs as fast as the parameter-space tile 229 in fp32 and a little
  slower in fp16, but it costs two launches per tunnel and step instead of two per step.

Either way every tunnel's populations are bit-identical to stepping its Solver alone, the
Solvers' ``cur`` is kept in sync, and ``event()`` orders later work after the steps. A
persistent batch must be rebuilt after any member Solver is stepped on its own.
"""
import ctypes

import torch

import wtlib as W
from wtlib import call, ptr


class MemberError(RuntimeError):
    """Some tunnels of a streams-executor step failed (``failed``: [(index, exception)]); every
    other tunnel was stepped as asked."""

    def __init__(self, failed):
        super().__init__('; '.join(f'tunnel {i}: {e}' for i, e in failed))
        self.failed = failed


class TunnelBatch:
    def __init__(self, solvers, params, tile=0, stream=None, mode='persistent'):
        if not solvers:
            raise ValueError('empty batch')
        if mode not in ('persistent', 'streams'):
            raise ValueError(f'unknown batch mode {mode!r}')
        self.mode = mode
        self.solvers = list(solvers)
        dev = self.solvers[0].dev
        for s in self.solvers:
            if s.dev != dev or s.precision != self.solvers[0].precision or s.collision != self.solvers[0].collision:
                raise ValueError('a batch needs one device, precision and collision form')
        self.dev = dev
        self.stream = stream if stream is not None else torch.cuda.Stream(dev)
        self.sh = W.stream_handle(self.stream)
        n = len(self.solvers)
        self.grids = (W.Grid * n)(*[s.grid for s in self.solvers])
        dbl = ctypes.c_double * n
        self._uin = dbl(*[float(p['uIn']) for p in params])
        self._tau = dbl(*[float(p['tau']) for p in params])
        self._smag = dbl(*[float(p['smag']) for p in params])
        self._cur = (ctypes.c_int32 * n)(*[s.cur for s in self.solvers])
        self.tile = int(tile)
        # per-tunnel step counts in one batch: the parameter-space tiles (tile 0 is one of them)
        self.steps_each = self.tile == 0 or self.tile // 100 == 2
        self.params = [dict(p) for p in params]
        self.cells = sum(s.n for s in self.solvers)
        self.handle = ctypes.c_void_p()
        if mode == 'streams':
            return
        nbytes = W.lib().wt_batch_workspace_bytes(self.grids, n, self.tile)
        if nbytes < 0:
            W.check(int(nbytes))
        for s in self.solvers:  # the member tunnels' pending work comes first
            self.stream.wait_stream(s.stream)
        with torch.cuda.stream(self.stream):
            self.workspace = torch.empty(int(nbytes), dtype=torch.uint8, device=dev)
        call('wt_batch_create', self.grids, n, self._uin, self._tau, self._smag, self._cur, self.tile,
             ptr(self.workspace), int(nbytes), self.sh, ctypes.byref(self.handle))

    def _sync_cur(self):
        cur = (ctypes.c_int32 * len(self.solvers))()
        call('wt_batch_cur', self.handle, cur)
        for s, c in zip(self.solvers, cur):
            s.cur = int(c)

    def _wait_members(self):
        # work queued on the member Solvers' own streams (frame kernels reading the
        # populations and mac) comes before the batch overwrites them
        for s in self.solvers:
            self.stream.wait_stream(s.stream)

    def _step_streams(self, steps, mac_all_last):
        # every member waits for the batch stream's earlier work, steps on its own stream,
        # and the batch stream waits for all of them
        start = torch.cuda.Event()
        start.record(self.stream)
        flags = W.STEP_MAC_ALL_LAST if mac_all_last else 0
        failed = []
        for j, (s, p, k) in enumerate(zip(self.solvers, self.params, steps)):
            if k <= 0:
                continue
            s.stream.wait_event(start)
            try:
                call('wt_step', s.gp, s.cur, int(k), float(p['uIn']), float(p['tau']), float(p['smag']), flags, s.sh)
            except W.WtError as e:  # this tunnel only; the others still step
                failed.append((j, e))
                continue
            s.cur ^= int(k) & 1
        self._wait_members()
        if failed:
            raise MemberError(failed)

    def step(self, steps, mac_all_last=True):
        """Advance every tunnel `steps` steps; `steps` may also be one count per tunnel with the
        streams executor (each tunnel is its own launch) and with a parameter-space tile
        (200 + k: each step launches the tunnels with steps to go)."""
        each = isinstance(steps, (list, tuple))
        if each:
            if len(steps) != len(self.solvers):
                raise ValueError('one step count per tunnel')
            counts = [int(k) for k in steps]
            if self.mode != 'streams' and len(set(counts)) > 1 and not self.steps_each:
                raise ValueError(f'batched tile {self.tile} steps every tunnel alike (a 200 + k tile does not)')
        else:
            counts = [int(steps)] * len(self.solvers)
        if self.mode == 'streams':
            self._step_streams(counts, mac_all_last)
            return
        self._wait_members()
        flags = W.STEP_MAC_ALL_LAST if mac_all_last else 0
        if each:
            call('wt_batch_step_each', self.handle, (ctypes.c_int32 * len(counts))(*counts), flags, self.sh)
        else:
            call('wt_batch_step', self.handle, counts[0], flags, self.sh)
        self._sync_cur()

    def _capture_streams(self, steps, mac_all_last):
        # the batch stream forks to every member stream and joins back inside one graph; an
        # even step count returns every tunnel to the buffer it started from, so replays chain
        if steps <= 0 or steps % 2:
            raise ValueError('capture needs an even, positive step count')
        self._wait_members()
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        flags = W.STEP_MAC_ALL_LAST if mac_all_last else 0
        with torch.cuda.graph(g, stream=self.stream):
            start = torch.cuda.Event()
            start.record(self.stream)
            for s, p in zip(self.solvers, self.params):
                s.stream.wait_event(start)
                call('wt_step', s.gp, s.cur, int(steps), float(p['uIn']), float(p['tau']), float(p['smag']), flags,
                     s.sh)
            for s in self.solvers:
                self.stream.wait_stream(s.stream)
        self._graph = g

    def capture(self, steps, mac_all_last=True):
        if self.mode == 'streams':
            self._capture_streams(steps, mac_all_last)
            return
        call('wt_batch_capture', self.handle, int(steps), W.STEP_MAC_ALL_LAST if mac_all_last else 0, self.sh)

    def replay(self):
        self._wait_members()
        if self.mode == 'streams':
            if getattr(self, '_graph', None) is None:
                raise RuntimeError('replay before capture')
            with torch.cuda.stream(self.stream):
                self._graph.replay()
            return
        call('wt_batch_replay', self.handle, self.sh)

    def event(self, timing=False):
        """A CUDA event recorded after the work queued so far on the batch stream; member
        Solvers wait on it (Solver.wait_event) before their frame kernels. With timing, two
        such events give the device time between them (Event.elapsed_time)."""
        e = torch.cuda.Event(enable_timing=timing)
        e.record(self.stream)
        return e

    def synchronize(self):
        self.stream.synchronize()

    def close(self):
        if self.mode == 'streams':
            self.stream.synchronize()
            self._graph = None
            return
        if self.handle:
            self.stream.synchronize()
            W.lib().wt_batch_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
