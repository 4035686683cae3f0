"""Multi-session serving loop: the reference's Engine thread (server/app.py:150-202) turned
into a request loop with continuous batching.

The reference runs one tunnel shared by every client, steps it from a 60 Hz loop and sends a
frame to the clients whose previous frame has been acknowledged (`ready`). Here each session
owns a tunnel on one GPU:

* **Admission.** A session is admitted in arrival order once its device footprint
  (``lbm.estimate_bytes``: populations, mac, mask, particle and frame buffers) fits in what
  the HBM budget has left. Later arrivals queue behind it. A session whose lifetime ends
  while it still waits leaves the queue (counted as abandoned).
* **Requests.** A session's client asks for its first frame on admission and for each next
  one when it has its previous frame and its 1/fps tick has come: the reference's `ready`
  flow control (server/app.py:173-193) with 30 fps pacing.
* **Rounds.** A round takes every session with an outstanding request. Their tunnels advance
  ``steps_per_frame`` steps together in one ``TunnelBatch``: by default each tunnel's own
  kernel on its own stream, all running at once (``batch_mode='streams'``), or one persistent
  bulk kernel per step over a tile work-list spanning every tunnel (``'persistent'``); the
  batch is rebuilt only when the set of sessions changes. Then each session's stream waits for the
  batch, advects its particles and runs its frame kernels, which write the wire-format frame
  straight into one device buffer (``Solver.launch_frame_packed``), and one copy brings it
  back. Frames are collected in session order. Sessions admitted while a round runs join
  the next round, so their work overlaps everyone else's from then on.
* **Commands.** ``command(session, msg, payload)`` takes a client's messages as the Engine's
  handle() does (server/app.py:104-149): 'params' (flow parameters, particle count,
  'running', 'steps', 'cp'), 'respawn', 'reset', 'ready' and the 'solid' / 'surface' uploads
  (checked by wire.upload_arrays). They run in arrival order when the next round starts. A
  paused session is not stepped and gets frames at 12 Hz; with the streams executor each
  session steps its own 'steps' per frame; surface pressure comes every third frame when
  'cp' is on (server/app.py:177-178). With ``pacing='client'`` a session's next frame waits for
  its client's 'ready', as in the reference; the default ``'fps'`` stands in for clients that
  acknowledge at once and ask again at their next 1/fps tick. ``disconnect(session)`` ends a
  session whose client has gone.
* **Failures.** A solver that cannot be created, or a session whose step, particles, frame or
  command raises, fails alone: it is reported in ``errors`` and the others are served.
* **Latency.** A frame's latency runs from its request to the moment its bytes are on the
  host. ``stats()`` gives p50/p99 over all frames, admitted/retired/abandoned/queued counts,
  the peak and end memory in use, and the aggregate lattice-update rate over the window.

Under oversubscription (more cells than the GPU can step at 30 x steps_per_frame per second)
every session is due in every round, frames come as fast as the GPU allows, and the frame
latency equals the round time: steps_per_frame x cells in service / throughput.
"""
import argparse
import collections
import heapq
import json
import time

import numpy as np

import bodies
import lbm
import wire
from batch import MemberError

PAUSED_HZ = 12  # frames per second of a paused session (server/app.py:20)
_SUBMIT = {'type': '_submit'}  # marks a session queued by enqueue() in the command deque


class Session:
    """One client's tunnel: its grid, mask and parameters (the Engine's `p` dict,
    server/app.py:61-63), its lifetime and its request clock."""

    def __init__(self, sid, dims, solid, params, lifetime, particles=5000, frontal=None, arrival=0.0):
        self.id = sid
        self.dims = tuple(int(d) for d in dims)
        nx, ny, nz = self.dims
        self.n = nx * ny * nz
        self.solid = solid
        self.p = dict(maxAge=2.2 * nx / (params['uIn'] * 10), lref=40.0, seedX=2.0, seedCy=(ny - 1) / 2,
                      seedCz=(nz - 1) / 2, seedHy=(ny - 4) / 2, seedHz=(nz - 4) / 2,
                      slice=dict(axis=1, index=ny // 2, field=0, vmin=0.0, vmax=1.6))
        self.p.update(params)
        self.particles = int(particles)
        self.lifetime = float(lifetime)
        self.arrival = float(arrival)
        self.frontal = frontal if frontal is not None else bodies.areas(solid, self.dims)[0]
        self.solver = None
        self.reuse = None          # a kept tunnel of this grid, re-initialised for this session
        self.bytes = 0
        self.request_t = None
        self.admitted_t = None
        self.last_t = None
        self.frames = 0
        self.steps = 0
        self.cd = self.cl = float('nan')
        self.last_frame = None
        self.mlups = 0.0
        self.frame_no = 0
        self.ready = True          # client pacing: the client holds no unacknowledged frame
        self.verts = self.norms = None  # surface points for Cp, once uploaded
        self.applied = []          # (frames before it, message, payload) per command, with keep_frames
        self.deferred = []         # commands that arrived while its tunnel was being built
        self.demand = 0.0          # lattice updates per second it requests (admission's work bound)

    @property
    def running(self):
        return bool(self.p.get('running', True))


class SessionServer:
    """Admission, rounds and latency accounting for many sessions on one GPU.

    ``solver_factory(session)`` returns a ready Solver (mask, equilibrium, particles) and
    ``batch_factory(solvers, params)`` a TunnelBatch; ``footprint(session)`` the bytes
    admission charges. The defaults build lbm.Solver / batch.TunnelBatch on ``device``.
    ``clock`` is the time source (seconds)."""

    def __init__(self, device='cuda:0', budget_bytes=160e9, precision='fp32', fps=30.0, steps_per_frame=10,
                 tile=0, collision=None, clock=time.perf_counter, solver_factory=None, batch_factory=None,
                 footprint=None, keep_frames=False, batch_mode='streams', pacing='fps', paused_hz=PAUSED_HZ,
                 rate_in_header=True, priorities=True, work_bound_glups=None, admit_thread=False, recycle=True,
                 new_per_round=None, arena=None):
        self.device = device
        self.budget = float(budget_bytes)
        self.precision = precision
        self.collision = collision
        self.period = 1.0 / fps
        self.steps_per_frame = int(steps_per_frame)
        # batched tile of the library executor: the parameter-space form of the two-cell tile
        # with early pulls (229; 204, at 128 registers, for fp64), the fastest batched shape on
        # config 4, which also steps sessions by their own counts
        self.tile = int(tile) if tile else (204 if precision == 'fp64' else 229)
        # executor of the round's steps: every tunnel's own kernel on its own stream, all at
        # once ('streams'), or the library's batched kernels ('persistent': two launches per
        # step for all sessions)
        self.batch_mode = batch_mode
        self.steps_each = batch_mode == 'streams' or self.tile // 100 == 2
        self.clock = clock
        self.solver_factory = solver_factory or self._make_solver
        # the default factory's tunnels are allocated on the serving thread at admission, when
        # the GPU is idle between rounds (an allocator that frees its cache synchronises the
        # device, and allocation holds driver locks), and initialised on the worker thread
        self._allocate = self._alloc_solver if solver_factory is None else None
        # arena: the default factory's tunnels take their per-cell state from one block of device
        # memory the size of the budget (arena.py), allocated at the first admission, so that
        # admitting and dropping tunnels makes no CUDA allocation; on by default with it
        self.use_arena = (solver_factory is None) if arena is None else bool(arena)
        self._arena = None
        self._released = collections.deque()  # tunnels a failed build left, to give back
        self.arena_waits = 0
        self.batch_factory = batch_factory or self._make_batch
        self.footprint = footprint or (lambda s: lbm.estimate_bytes(s.dims, precision, s.particles))
        self.keep_frames = keep_frames
        # 'fps': each client asks for its next frame at its next 1/fps tick (the simulated
        # clients of config 5); 'client': only after it acknowledges the last one ('ready')
        if pacing not in ('fps', 'client'):
            raise ValueError(f'unknown pacing {pacing!r}')
        self.pacing = pacing
        self.paused_period = 1.0 / paused_hz
        self.rate_in_header = rate_in_header
        # streams executor: each session's stream gets a CUDA priority by tunnel size, smaller
        # tunnels higher, so within a round their few blocks are scheduled ahead of the big
        # tunnels' and their frames finish early; every session still gets one frame per round
        self.priorities = priorities
        # opt-in admission bound on requested work: admit a session only while the lattice
        # updates per second that every admitted session requests (cells x steps per frame x
        # fps) stay within work_bound_glups; None admits by the HBM budget alone
        self.work_bound = None if work_bound_glups is None else float(work_bound_glups) * 1e9
        self.demand = 0.0
        # admit_thread: a worker thread initialises admitted sessions' tunnels (mask upload,
        # codes, link list, equilibrium, particles) while rounds run, after admission has
        # allocated them or taken kept ones; a session joins the first round after its tunnel
        # is ready, and commands sent meanwhile wait for it. Without it (the default) admission
        # builds the tunnel inside the round.
        # recycle: a retired session's tunnel (when its solver has recycle()) is kept, its bytes
        # still charged to the budget, for the next session of the same grid, precision and
        # collision form, which re-initialises it instead of allocating; admission evicts kept
        # tunnels of other grids when it needs their memory
        self.recycle = recycle
        # new_per_round: at most this many tunnels are newly allocated per round (kept tunnels
        # are not counted); allocating several large tunnels at once under a nearly full
        # budget can take the allocator hundreds of milliseconds, all of it in one round
        self.new_per_round = new_per_round
        self._pool = {}                     # (dims, particles) -> [(solver, bytes)] kept tunnels
        self.pooled = 0.0
        self.pool_hits = self.pool_evictions = 0
        self.building = {}                  # id -> Session whose tunnel the worker is building
        self._built = collections.deque()   # (session, exception or None) the worker finished
        self._jobs = None
        if admit_thread:
            self._start_worker()
        # (session id, message, payload) in arrival order; a deque, so the front end's threads
        # can append while the serving thread drains (the reference's handlers feed its Engine
        # through a queue the same way, server/app.py:212-222)
        self._cmds = collections.deque()
        self.round_frames = []    # (session id, frame bytes) produced by the latest round
        self.active = {}          # id -> Session, in admission order
        self.queue = []           # FIFO of sessions waiting for memory
        self.used = 0.0
        self.peak_used = 0.0
        self.latencies = []
        self.frame_log = []       # (session id, frame bytes) when keep_frames
        self.cell_updates = 0
        self.t0 = None
        self.rounds = 0
        self.rebuilds = 0
        self.max_active = 0
        self.active_sum = 0
        self.max_queued = 0
        self.admitted = self.retired = self.abandoned = self.failed = 0
        self.errors = []          # (session id, message) for the sender: the Engine's 'error' JSON
        self._batch = None
        self._batch_key = None
        self._stream = None
        self.phase = {'admit': 0.0, 'rebuild': 0.0, 'issue': 0.0, 'collect': 0.0}
        self.round_s = []
        # per round: (wall s, device s of the batched steps, sessions due, cell updates, tunnels
        # that joined, tunnels still being built, sessions retired before it, issue s, collect s)
        self.round_log = []
        self.step_gpu_s = 0.0  # device time of the batched steps (CUDA events on the batch stream)
        self.step_cells = 0

    def _start_worker(self):
        import queue
        import threading
        self._jobs = queue.Queue()

        def work():
            if self.device is not None:
                import torch
                torch.cuda.set_device(torch.device(self.device))
            while True:
                s = self._jobs.get()
                if s is None:
                    return
                try:
                    s.solver, err = self.solver_factory(s), None
                except Exception as e:  # reported by the serving thread (server/app.py:115-122)
                    s.solver, err = None, e
                self._built.append((s, err))
        self._worker = threading.Thread(target=work, name='admission', daemon=True)
        self._worker.start()

    # ---- default factories (the GPU path) ----
    def _priority(self, s):
        """CUDA stream priority of a session (lower is higher): smaller tunnels first."""
        if not self.priorities or self.batch_mode != 'streams':
            return 0
        return -3 if s.n <= 1_000_000 else (-2 if s.n <= 4_000_000 else (-1 if s.n <= 16_000_000 else 0))

    def _arena_get(self):
        if self._arena is None:
            import arena
            self._arena = arena.Arena(self.budget, self.device)
        return self._arena

    def _state_bytes(self, s):
        return lbm.state_layout(s.dims, self.precision)[1]

    def _drop_solver(self, sv):
        """A tunnel leaves for good: its arena range goes back."""
        off = getattr(sv, 'arena_off', None)
        if off is not None:
            self._arena.release(off)
            sv.arena_off = None

    def _alloc_solver(self, s):
        """A new tunnel's device and pinned frame buffers (lbm.Solver), on its own stream, its
        per-cell state in a range of the arena when the server uses one."""
        import torch
        off, storage = None, None
        if self.use_arena:
            a = self._arena_get()
            total = self._state_bytes(s)
            off = a.alloc(total)
            if off is None:
                raise MemoryError(f'no free range of {total} bytes in the tunnel arena')
            storage = a.view(off, total)
        try:
            stream = torch.cuda.Stream(torch.device(self.device), priority=self._priority(s))
            sv = lbm.Solver(s.dims, self.device, precision=self.precision, collision=self.collision, seed=s.id,
                            stream=stream, storage=storage)
            sv.prepare_frame(s.p, s.verts is not None)
        except Exception:
            if off is not None:
                self._arena.release(off)
            raise
        sv.arena_off = off
        sv.fresh = True
        return sv

    def _make_solver(self, s):
        if s.reuse is not None:  # a kept tunnel of this grid, or one allocated at admission
            sv, s.reuse = s.reuse, None
        else:
            sv = self._alloc_solver(s)
        try:
            if not getattr(sv, 'fresh', False):
                sv.recycle(seed=s.id)
            sv.fresh = False
            sv.set_solid(s.solid)
            sv.reset(s.p['uIn'])
            if s.particles:
                sv.set_particles(s.particles, s.p)
            if s.verts is not None:
                sv.set_surface(s.verts, s.norms)
            sv.prepare_frame(s.p, s.verts is not None)
            sv.synchronize()
        except Exception:
            self._released.append(sv)  # the serving thread gives its arena range back
            raise
        return sv

    def _make_batch(self, solvers, params):
        import torch
        from batch import TunnelBatch
        if self._stream is None:
            self._stream = torch.cuda.Stream(torch.device(self.device))
        return TunnelBatch(solvers, params, tile=self.tile, stream=self._stream, mode=self.batch_mode)

    # ---- client commands (server/app.py:104-149, one session each) ----
    def command(self, sid, msg, payload=None):
        """Queue a client's command for its session: the JSON messages 'params', 'respawn',
        'reset' and 'ready', or an upload 'solid' / 'surface' with its gzip payload (the two
        halves wire.decode_upload returns). Commands run in arrival order at the start of the
        next round, as the reference's Engine drains its queue before it steps. A session still
        waiting for memory keeps its parameters and uploads for when it is admitted. A
        resolution change ('grid') is a new session: its footprint goes through admission.
        command() and disconnect() may be called from other threads (a WebSocket front end's
        handlers) while the serving thread runs rounds; a session queued from such a thread
        goes through enqueue(), so that its commands cannot overtake it. A command for a
        session that is not (or no longer) here is reported in ``errors``."""
        if msg.get('type') == 'grid':
            raise ValueError("a resolution change is a new session; submit one")
        self._cmds.append((sid, dict(msg), payload))

    def fits(self, dims, particles=5000):
        """Whether a session of this grid can ever be admitted: its footprint within the HBM
        budget. The Engine's fits() (server/app.py:71-75) asks the same of a resolution before
        it builds a Solver, and answers 'does not fit on this device' otherwise."""
        return self.footprint(Session(-1, dims, None, dict(uIn=0.05, tau=0.51, smag=0.16), 0.0,
                                      particles=particles, frontal=1)) <= self.budget

    def disconnect(self, sid):
        """The session's client has gone (its WebSocket closed): at the next round an admitted
        session is retired and its memory released, and one still waiting leaves the queue."""
        self._cmds.append((sid, None, None))

    def _invalidate(self, s):
        # a batched tunnel's parameters, buffers or mask changed: rebuild the batch
        if self._batch is not None and self._batch_key is not None and s.id in self._batch_key:
            self._batch.close()
            self._batch, self._batch_key = None, None

    def _apply_commands(self, now):
        for _ in range(len(self._cmds)):  # those queued before this round; later ones wait
            sid, msg, payload = self._cmds.popleft()
            if msg is _SUBMIT:
                self.submit(payload)
                continue
            if sid in self.building:  # its tunnel is being built: applied once it is active
                self.building[sid].deferred.append((msg, payload))
                continue
            s = self.active.get(sid)
            if s is None:
                s = next((q for q in self.queue if q.id == sid), None)
            if s is None:
                # gone (retired, failed, disconnected) or never here: the reference ignores
                # commands without a solver; a command, unlike a late disconnect, is reported
                if msg is not None:
                    self.errors.append((sid, f"command {msg.get('type')!r} for no session"))
                continue
            self._apply_one(s, msg, payload, now)

    def _apply_one(self, s, msg, payload, now):
        if msg is None:  # disconnected: the lifetime ends now (retired or abandoned)
            s.lifetime = min(s.lifetime, now - s.arrival)
            return
        if self.keep_frames:  # which frames each command came before (test replays)
            s.applied.append((s.frame_no, dict(msg), payload))
        try:
            self._apply(s, msg, payload, now)
        except Exception as e:  # a bad message fails alone (the Engine reports it, server/app.py:160-161)
            self.errors.append((s.id, f'command failed: {e!r}'))

    def _apply(self, s, msg, payload, now):
        t = msg.get('type')
        sv = s.solver
        if t == 'ready':
            if not s.ready:
                s.ready = True
                s.request_t = now
        elif t == 'params':
            old = int(s.p.get('particles', s.particles))
            s.p.update({k: v for k, v in msg.items() if k != 'type'})
            new = int(s.p.get('particles', old))
            # a new count re-seeds only a tunnel that has particles (server/app.py:128-131)
            if new != old and (sv.num_p if sv is not None else s.particles):
                s.particles = new
                if sv is not None:
                    sv.set_particles(new, s.p)
            self._invalidate(s)
        elif t == 'respawn':
            if sv is not None:
                sv.set_particles(int(s.p.get('particles', s.particles)), s.p)
            else:  # still waiting for memory: the tunnel gets its particles when it is created
                s.particles = int(s.p.get('particles', s.particles))
        elif t == 'reset':
            if sv is not None:
                self._invalidate(s)
                sv.reset(s.p['uIn'])
        elif t in ('solid', 'surface'):
            got = wire.upload_arrays(msg, payload, s.dims)
            if got is None:
                return
            if got[0] == 'solid':
                s.solid = got[1].copy()
                s.frontal = bodies.areas(s.solid, s.dims)[0]
                if sv is not None:
                    self._invalidate(s)
                    sv.set_solid(s.solid)
            else:
                s.verts, s.norms = got[1].copy(), got[2].copy()
                if sv is not None:
                    sv.set_surface(s.verts, s.norms)

    def _frame_steps(self, s):
        """Steps before a session's next frame: none while paused; its own 'steps' with the
        streams executor (each tunnel its own launch) and the parameter-space batched tiles
        (200 + k, each step launching the tunnels with steps to go); the server's
        steps_per_frame with the work-list forms (one launch steps every tunnel alike)."""
        if not s.running:
            return 0
        if self.steps_each:
            return int(s.p.get('steps', self.steps_per_frame))
        return self.steps_per_frame

    def _due(self, s, now):
        if self.pacing == 'client':
            return s.ready and (s.running or now - s.last_t >= self.paused_period)
        return s.request_t <= now

    def _want_cp(self, s):
        # the Engine's surface pressure cadence (server/app.py:177-178)
        every = max(3, s.solver.num_verts // 20000)
        return bool(s.p.get('cp')) and s.solver.num_verts > 0 and s.frame_no % every == 0

    # ---- admission ----
    def submit(self, session):
        """Queue a session for admission now (the serving thread, or a single-threaded
        driver)."""
        self.queue.append(session)
        self.max_queued = max(self.max_queued, len(self.queue))

    def enqueue(self, session):
        """Queue a session from another thread (a front end's handler): it joins the admission
        queue when the next round starts, in order with the commands queued after it, so a
        command sent right after enqueue() finds its session."""
        self._cmds.append((session.id, _SUBMIT, session))

    def _activate(self, s, now):
        s.bytes = max(s.bytes, s.solver.device_bytes())
        s.admitted_t = s.request_t = s.last_t = now
        self.active[s.id] = s
        self.admitted += 1

    def _admit(self, now):
        allocated = 0
        while self._released:
            self._drop_solver(self._released.popleft())
        while self._built:  # tunnels the worker finished join this round
            s, err = self._built.popleft()
            del self.building[s.id]
            if err is not None:
                self.used -= s.bytes
                self.demand -= s.demand
                self.failed += 1
                self.errors.append((s.id, f'Could not allocate {"x".join(map(str, s.dims))} grid: {err}'))
                continue
            self.used -= s.bytes
            self._activate(s, now)
            self.used += s.bytes
            self.peak_used = max(self.peak_used, self.used + self.pooled)
            for msg, payload in s.deferred:  # commands sent while it was being built
                self._apply_one(s, msg, payload, now)
            s.deferred = []
        while self.queue:
            s = self.queue[0]
            if now - s.arrival >= s.lifetime:  # the client gave up while waiting
                self.queue.pop(0)
                self.abandoned += 1
                continue
            need = self.footprint(s)
            key = self._pool_key(s)
            kept = self._pool.get(key)
            if not kept and self.new_per_round is not None and allocated >= self.new_per_round:
                break  # the next round allocates it
            if not kept and self.use_arena and self._allocate is not None:
                total = self._state_bytes(s)
                if self._arena_get().largest() < total:  # kept tunnels give their ranges back
                    self._evict_for_range(total)
                    if self._arena.largest() < total:
                        self.arena_waits += 1
                        break
            reuse_bytes = kept[-1][1] if kept else 0.0
            over = self.used + self.pooled - reuse_bytes + max(need, reuse_bytes) - self.budget
            if over > 0:  # drop kept tunnels, never the one this session would take
                self._evict(over, spare=key if kept else None)
                if self.used + self.pooled - reuse_bytes + max(need, reuse_bytes) > self.budget:
                    break
            want = self._demand(s)
            if self.work_bound is not None and self.active and self.demand + want > self.work_bound:
                break
            self.queue.pop(0)
            if kept:  # the kept tunnel of this grid leaves the pool for this session
                s.reuse, b = kept.pop()
                if not kept:
                    del self._pool[key]
                self.pooled -= b
                need = max(need, b)
                self.pool_hits += 1
            s.demand = want
            if not kept:
                allocated += 1
            if self._jobs is not None:  # built by the worker; memory and demand reserved now
                if s.reuse is None and self._allocate is not None:
                    try:
                        s.reuse = self._allocate(s)
                    except Exception as e:  # out of memory etc. (server/app.py:115-122)
                        self.failed += 1
                        self.errors.append((s.id, f'Could not allocate {"x".join(map(str, s.dims))} grid: {e}'))
                        continue
                s.bytes = need
                self.used += need
                self.demand += want
                self.peak_used = max(self.peak_used, self.used + self.pooled)
                self.building[s.id] = s
                self._jobs.put(s)
                continue
            try:
                s.solver = self.solver_factory(s)
            except Exception as e:  # out of memory etc. (server/app.py:115-122)
                s.solver = None
                self.failed += 1
                self.errors.append((s.id, f'Could not allocate {"x".join(map(str, s.dims))} grid: {e}'))
                continue
            s.bytes = need
            self._activate(s, now)
            self.demand += want
            self.used += s.bytes
            self.peak_used = max(self.peak_used, self.used + self.pooled)
        self.max_active = max(self.max_active, len(self.active))

    def _demand(self, s):
        """Lattice updates per second the session requests: cells x steps per frame x fps."""
        return s.n * int(s.p.get('steps', self.steps_per_frame)) / self.period

    def _fail(self, s, err):
        """A session whose tunnel raised: reported, retired, its memory released; the others
        go on (the reference's Engine prints a solver error and keeps serving)."""
        self._invalidate(s)
        self.active.pop(s.id, None)
        self.used -= s.bytes
        self.demand -= getattr(s, 'demand', 0.0)
        try:
            s.solver.synchronize()
        except Exception:
            pass
        self._drop_solver(s.solver)
        s.solver = None
        self.failed += 1
        self.errors.append((s.id, f'solver error: {err!r}'))

    def _retire(self, now):
        gone = [s for s in self.active.values() if now - s.arrival >= s.lifetime]
        if not gone:
            return
        if self._batch is not None and any(s.id in self._batch_key for s in gone):
            self._batch.close()
            self._batch, self._batch_key = None, None
        for s in gone:
            del self.active[s.id]
            self.used -= s.bytes
            self.demand -= getattr(s, 'demand', 0.0)
            s.solver.synchronize()
            if self.recycle and hasattr(s.solver, 'recycle'):
                self._pool.setdefault(self._pool_key(s), []).append((s.solver, s.bytes))
                self.pooled += s.bytes
            else:
                self._drop_solver(s.solver)
            s.solver = None
            self.retired += 1

    def _pool_key(self, s):
        return tuple(s.dims)  # precision and collision form are the server's

    def _evict(self, need, spare=None):
        """Drop kept tunnels, the largest first, until `need` bytes are free; the last kept
        tunnel of grid `spare` (the one an arriving session takes) stays."""
        order = sorted(((k, j) for k, v in self._pool.items() for j in range(len(v))
                        if not (k == spare and j == len(v) - 1)),
                       key=lambda kj: -self._pool[kj[0]][kj[1]][1])
        drop = []
        for k, j in order:
            if need <= 0:
                break
            need -= self._pool[k][j][1]
            drop.append((k, j))
        for k, j in sorted(drop, key=lambda kj: -kj[1]):
            sv, b = self._pool[k].pop(j)
            self._drop_solver(sv)
            self.pooled -= b
            self.pool_evictions += 1
            if not self._pool[k]:
                del self._pool[k]

    def _evict_for_range(self, total):
        """Drop kept tunnels, the largest first, until the arena has a free range of `total`
        bytes."""
        while self._pool and self._arena.largest() < total:
            k, j = max(((k, j) for k, v in self._pool.items() for j in range(len(v))),
                       key=lambda kj: self._pool[kj[0]][kj[1]][1])
            sv, b = self._pool[k].pop(j)
            self._drop_solver(sv)
            self.pooled -= b
            self.pool_evictions += 1
            if not self._pool[k]:
                del self._pool[k]

    # ---- one round ----
    def round(self):
        """Retire, admit, then serve every session with an outstanding request, oldest request
        first, and collect the frames as they complete. Returns the number of frames produced."""
        now = self.clock()
        if self.t0 is None:
            self.t0 = now
        self.round_frames = []  # (session id, frame bytes) of this round, for the sender
        self._apply_commands(now)
        retired0, joined0 = self.retired, self.admitted
        self._retire(now)
        self._admit(now)
        retired, joined = self.retired - retired0, self.admitted - joined0
        t_admit = self.clock()
        due = sorted((s for s in self.active.values() if self._due(s, now)), key=lambda s: s.request_t)
        self.max_active = max(self.max_active, len(self.active))
        if not due:
            self.phase['admit'] += t_admit - now
            return 0
        ks = {s.id: self._frame_steps(s) for s in due}
        # the batch holds its tunnels in id order, so the order of requests never rebuilds it
        stepping = sorted((s for s in due if ks[s.id] > 0), key=lambda s: s.id)
        started = done = None
        if stepping:
            key = tuple(s.id for s in stepping)
            if key != self._batch_key:
                if self._batch is not None:
                    self._batch.close()
                self._batch = self.batch_factory([s.solver for s in stepping], [s.p for s in stepping])
                self._batch_key = key
                self.rebuilds += 1
        t_rebuild = self.clock()
        broken = {}
        if stepping:
            counts = [ks[s.id] for s in stepping]
            started = self._batch.event(timing=True)
            try:
                self._batch.step(counts[0] if len(set(counts)) == 1 else counts)
            except MemberError as e:
                broken.update((stepping[j].id, err) for j, err in e.failed)
            done = self._batch.event(timing=True)
        for s in due:
            if s.id in broken:
                continue
            k = ks[s.id]
            try:
                if k:
                    # the streams executor stepped this tunnel on its own stream, which orders
                    # its frame after its own steps; the persistent one steps all at once
                    if self.batch_mode != 'streams':
                        s.solver.wait_event(done)
                    s.solver.advance_particles(k, s.p)
                s.frame_no += 1
                s.solver.launch_frame_packed(s.p, self._want_cp(s))
            except Exception as e:
                broken[s.id] = e
        t_issue = self.clock()
        pending = [s for s in due if s.id not in broken]
        while pending:  # frames in the order they complete
            ready = [s for s in pending if s.solver.frame_ready()]
            if not ready:
                time.sleep(20e-6)
                continue
            for s in ready:
                pending.remove(s)
                self._collect(s, ks[s.id], broken)
        for s in due:
            if s.id in broken:
                self._fail(s, broken[s.id])
        t_end = self.clock()
        step_s, cells = 0.0, 0
        if started is not None:  # every frame has been collected, so both events are complete
            done.synchronize()
            step_s = started.elapsed_time(done) / 1e3
            cells = sum(s.n * ks[s.id] for s in stepping if s.id not in broken)
            self.step_gpu_s += step_s
            self.step_cells += cells
        self.round_log.append((t_end - now, step_s, len(due), cells, joined, len(self.building), retired,
                               t_issue - t_rebuild, t_end - t_issue))
        for name, a, b in (('admit', now, t_admit), ('rebuild', t_admit, t_rebuild), ('issue', t_rebuild, t_issue),
                           ('collect', t_issue, t_end)):
            self.phase[name] += b - a
        self.round_s.append(t_end - now)
        self.rounds += 1
        self.active_sum += len(self.active)
        return len(due) - len(broken)

    def _collect(self, s, k, broken):
        """Take a session's finished frame: header, latency, the client's Cd/Cl and request."""
        sv = s.solver
        header = dict(type='frame', dims=list(s.dims), numP=sv.num_p, numVerts=sv.num_verts, forces=None, steps=k,
                      mlups=s.mlups if (self.rate_in_header and s.running) else 0.0, running=s.running)
        t_prev = s.last_t
        try:
            frame = sv.collect_frame_packed(header)
        except Exception as e:
            broken[s.id] = e
            return
        t = self.clock()
        self.latencies.append(t - s.request_t)
        self.round_frames.append((s.id, frame))
        if self.keep_frames:
            self.frame_log.append((s.id, frame))
        s.last_frame = frame
        s.frames += 1
        s.steps += k
        s.last_t = t
        self.cell_updates += s.n * k
        fx, fy = float(sv.last_forces6[0]), float(sv.last_forces6[1])
        q = 0.5 * s.p['uIn'] ** 2 * max(1, s.frontal)  # the client's Cd/Cl (web/js/main.js:337-339)
        s.cd, s.cl = fx / q, fy / q
        s.mlups = s.n * k / max(1e-9, t - t_prev) / 1e6
        if self.pacing == 'client':
            s.ready = False  # until the client acknowledges this frame
        else:
            # the client acknowledges at once and asks again at its next tick
            s.request_t = max(t, s.request_t + (self.period if s.running else self.paused_period))

    def stats(self):
        now = self.clock()
        lat = np.array(self.latencies) * 1e3 if self.latencies else np.zeros(1)
        rs = np.array(self.round_s) * 1e3 if self.round_s else np.zeros(1)
        span = max(1e-9, now - (self.t0 if self.t0 is not None else now))
        return {'frames': len(self.latencies), 'p50_ms': round(float(np.percentile(lat, 50)), 2),
                'p99_ms': round(float(np.percentile(lat, 99)), 2), 'max_ms': round(float(lat.max()), 2),
                'rounds': self.rounds, 'batch_rebuilds': self.rebuilds, 'admitted': self.admitted,
                'retired': self.retired, 'abandoned': self.abandoned, 'failed': self.failed,
                'active_end': len(self.active), 'building_end': len(self.building),
                'max_active': self.max_active,
                'mean_active': round(self.active_sum / max(1, self.rounds), 1), 'queued_end': len(self.queue),
                'max_queued': self.max_queued, 'used_gb_end': round(self.used / 1e9, 2),
                'kept_gb_end': round(self.pooled / 1e9, 2), 'tunnels_reused': self.pool_hits,
                'kept_tunnels_dropped': self.pool_evictions,
                'arena_gb': None if self._arena is None else round(self._arena.size / 1e9, 2),
                'arena_largest_free_gb_end': None if self._arena is None else round(self._arena.largest() / 1e9, 2),
                'arena_waits': self.arena_waits,
                'peak_used_gb': round(self.peak_used / 1e9, 2),
                'glups': round(self.cell_updates / span / 1e9, 3),
                'step_glups_device': round(self.step_cells / max(1e-9, self.step_gpu_s) / 1e9, 3),
                'step_share_of_wall': round(self.step_gpu_s / span, 3),
                'round_ms': {'p50': round(float(np.percentile(rs, 50)), 1), 'p99': round(float(np.percentile(rs, 99)), 1),
                             **{f'{k}_mean': round(v / max(1, self.rounds) * 1e3, 2) for k, v in self.phase.items()}},
                'frames_per_session_s': round(len(self.latencies) / span / max(1e-9, self.active_sum / max(1, self.rounds)), 2),
                'requested_glups_end': round(self.demand / 1e9, 2),
                'work_bound_glups': None if self.work_bound is None else round(self.work_bound / 1e9, 2),
                'slow_rounds': self.slow_rounds()}

    def slow_rounds(self, k=8):
        """The k longest rounds of the window beside the median one: wall and device step time,
        sessions, cell updates and the device rate, tunnels that joined, tunnels still being
        built, sessions retired just before, and the host's issue and collect phases."""
        if not self.round_log:
            return []
        keys = ('ms', 'step_ms', 'sessions', 'gcells', 'joined', 'building', 'retired', 'issue_ms', 'collect_ms')
        order = sorted(range(len(self.round_log)), key=lambda i: self.round_log[i][0])
        pick = order[::-1][:k] + [order[len(order) // 2]]
        out = []
        for i in pick:
            r = self.round_log[i]
            d = dict(zip(keys, (round(r[0] * 1e3, 1), round(r[1] * 1e3, 1), r[2], round(r[3] / 1e9, 3), r[4], r[5],
                                r[6], round(r[7] * 1e3, 1), round(r[8] * 1e3, 1))))
            d['glups'] = round(r[3] / r[1] / 1e9, 2) if r[1] > 0 else None
            d['round'] = i
            out.append(d)
        out[-1]['median'] = True
        return out

    def reset_window(self):
        """Start a fresh measurement window (drop latencies and counters so far)."""
        self.latencies.clear()
        self.round_s.clear()
        self.round_log.clear()
        self.phase = dict.fromkeys(self.phase, 0.0)
        self.step_gpu_s = 0.0
        self.step_cells = 0
        self.cell_updates = 0
        self.rounds = self.active_sum = 0
        self.t0 = self.clock()

    def close(self):
        if self._jobs is not None:  # stop the admission worker once it has finished its tunnel
            self._jobs.put(None)
            self._worker.join()
            self._jobs = None
            while self._built:
                s, _ = self._built.popleft()
                if s.solver is not None:
                    s.solver.synchronize()
            self.building.clear()
        if self._batch is not None:
            self._batch.close()
            self._batch, self._batch_key = None, None
        for s in self.active.values():
            s.solver.synchronize()
        self.active.clear()
        self._pool.clear()
        self.pooled = 0.0
        if self._arena is not None:  # every tunnel is gone: the arena's memory goes back
            import torch
            self._arena = None
            torch.cuda.empty_cache()


# ---- config 5: Poisson arrivals of tunnels of four sizes ----
SIZES = {0.5e6: (128, 64, 64), 2e6: (200, 100, 100), 8e6: (320, 160, 160), 33.5e6: (512, 256, 256)}
PROBS = (0.4, 0.3, 0.2, 0.1)


def masks(per_size=2, seed=55):
    """Seeded ellipsoid-union obstacles (1-6 ellipsoids on a moving belt) for each size,
    with their frontal areas: {size: [(solid, frontal), ...]}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = {}
    for size, dims in SIZES.items():
        out[size] = []
        for _ in range(per_size):
            solid, _ = bodies.ellipsoid_union(dims, int(rng.integers(1, 7)), int(rng.integers(1 << 31)),
                                              scale=dims[0] / 512.0, floor='belt')
            out[size].append((solid, bodies.areas(solid, dims)[0]))
    return out


class Arrivals:
    """Session generator for config 5: sizes {0.5, 2, 8, 33.5}M cells with probabilities
    {0.4, 0.3, 0.2, 0.1}, u0 uniform in [0.03, 0.08], nu uniform in [0.001, 0.01]
    (tau = 3 nu + 1/2), Cs = 0.16, exponential lifetimes, all from one PCG64 stream."""

    def __init__(self, seed=5, mean_life=60.0, particles=5000, mask_set=None):
        self.rng = np.random.Generator(np.random.PCG64(seed))
        self.mean_life = mean_life
        self.particles = particles
        self.masks = mask_set if mask_set is not None else masks()
        self.sizes = list(SIZES)
        self.next_id = 0

    def session(self, now):
        size = self.sizes[int(self.rng.choice(len(self.sizes), p=PROBS))]
        dims = SIZES[size]
        solid, frontal = self.masks[size][self.next_id % len(self.masks[size])]
        u0 = float(self.rng.uniform(0.03, 0.08))
        nu = float(self.rng.uniform(0.001, 0.01))
        s = Session(self.next_id, dims, solid, dict(uIn=u0, tau=3 * nu + 0.5, smag=0.16),
                    lifetime=float(self.rng.exponential(self.mean_life)), particles=self.particles,
                    frontal=frontal, arrival=now)
        self.next_id += 1
        return s


def simulate(duration=300.0, rate=2.0, mean_life=60.0, budget=160e9, precision='fp32', seed=5, device='cuda:0',
             particles=5000, warm_start=True, tile=0, steps_per_frame=10, fps=30.0, mask_set=None, keep=None,
             before_window=None, latencies_out=None, server_factory=None, warmup_s=0.0, work_bound_glups=None,
             batch_mode='streams'):
    """Config 5 in wall-clock time: Poisson arrivals at `rate` per second for `duration`
    seconds, each session requesting `fps` frames per second of its particles, one slice and
    Cd/Cl, admitted against `budget` bytes. With warm_start the run begins from the arrival
    process's stationary population (Poisson with mean rate x mean_life sessions; lifetimes
    are memoryless, so their residual lifetimes are exponential with the same mean), so the
    window measures the steady state; the set-up of those sessions is not timed. ``warmup_s``
    seconds of rounds over those sessions (no arrivals, not timed) come before the window.

    For one GPU of several (placement.py): ``keep(session, t)`` is asked about every session
    of the arrival stream, t its arrival in seconds from the start of the window (0 for the
    stationary ones), and only the sessions it accepts are served here; ``before_window()``
    runs between the set-up and the window (a barrier across GPUs); ``latencies_out`` (a list)
    receives the window's frame latencies in seconds. ``server_factory`` replaces the
    SessionServer constructor (same arguments)."""
    gen = Arrivals(seed, mean_life, particles, mask_set)
    srv = (server_factory or SessionServer)(device, budget_bytes=budget, precision=precision, fps=fps,
                                            steps_per_frame=steps_per_frame, tile=tile, admit_thread=True,
                                            work_bound_glups=work_bound_glups, batch_mode=batch_mode, new_per_round=1)

    def offer(s, t):
        if keep is None or keep(s, t):
            srv.submit(s)

    start = time.perf_counter()
    if warm_start:
        for _ in range(int(gen.rng.poisson(rate * mean_life))):
            offer(gen.session(start), 0.0)
        srv._admit(start)
        while srv.building:  # the worker builds the stationary sessions' tunnels
            time.sleep(0.01)
            srv._admit(time.perf_counter())
        srv.round()  # the stationary sessions have been running: one round builds their batch
        t_warm = time.perf_counter()
        while time.perf_counter() - t_warm < warmup_s:
            if srv.round() == 0:
                time.sleep(0.0005)
    setup_s = time.perf_counter() - start
    if before_window is not None:
        before_window()
    t0 = time.perf_counter()
    for s in srv.active.values():  # the window starts now; set-up time is not service time
        s.arrival += t0 - start
        s.admitted_t = s.request_t = s.last_t = t0
    for s in srv.queue:
        s.arrival += t0 - start
    arrivals, t = [], t0
    while True:
        t += float(gen.rng.exponential(1.0 / rate))
        if t > t0 + duration:
            break
        heapq.heappush(arrivals, t)
    srv.reset_window()
    while time.perf_counter() < t0 + duration:
        now = time.perf_counter()
        while arrivals and arrivals[0] <= now:
            t = heapq.heappop(arrivals)
            offer(gen.session(t), t - t0)
        if srv.round() == 0:
            time.sleep(0.0005)
    out = srv.stats()
    out.update(precision=precision, duration_s=duration, arrival_rate=rate, mean_lifetime_s=mean_life,
               budget_gb=budget / 1e9, warm_start=warm_start, steps_per_frame=steps_per_frame, fps=fps,
               particles=particles, setup_s=round(setup_s, 1), warmup_s=warmup_s, batch_mode=batch_mode,
               tile=srv.tile if batch_mode != 'streams' else None)
    if latencies_out is not None:
        latencies_out.extend(srv.latencies)
    srv.close()
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description='Config 5 serving simulation (Poisson sessions on one GPU)')
    ap.add_argument('--duration', type=float, default=300.0)
    ap.add_argument('--rate', type=float, default=2.0)
    ap.add_argument('--mean-life', type=float, default=60.0)
    ap.add_argument('--budget-gb', type=float, default=160.0)
    ap.add_argument('--precision', nargs='+', default=['fp32', 'fp16'])
    ap.add_argument('--steps-per-frame', type=int, default=10)
    ap.add_argument('--tile', type=int, default=0)
    ap.add_argument('--seed', type=int, default=5)
    ap.add_argument('--warmup', type=float, default=3.0, help='untimed seconds of rounds before the window')
    ap.add_argument('--batch-mode', nargs='+', default=['streams'], choices=['streams', 'persistent'])
    ap.add_argument('--work-bound', type=float, default=None, help='admission bound on requested GLUPS')
    a = ap.parse_args(argv)
    ms = masks()
    for prec in a.precision:
        for mode in a.batch_mode:
            r = simulate(a.duration, a.rate, a.mean_life, a.budget_gb * 1e9, prec, a.seed, tile=a.tile,
                         steps_per_frame=a.steps_per_frame, mask_set=ms, warmup_s=a.warmup, batch_mode=mode,
                         work_bound_glups=a.work_bound)
            print(json.dumps(r), flush=True)


if __name__ == '__main__':
    main()
