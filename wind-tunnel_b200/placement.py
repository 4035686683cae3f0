"""Session placement over the GPUs of one node: independent sessions spread over the GPUs, with
no exchange between them. A tunnel stays on one GPU, as the reference keeps its one Solver on
one device (server/app.py:56, 116); what the reference's single Engine cannot do is run more
than one tunnel, so there is no reference placement rule to follow.

One process per GPU runs its own SessionServer. Every process sees the same arrival stream
(what a front end sees: a session's arrival, its grid, and its departure when the client
disconnects) and applies the same deterministic rule to it, so the processes agree on where
each session goes without talking to each other, and each serves only its own sessions.

Rule (least connected work that fits): a session arriving at time t goes to the GPU with the
fewest connected cells -- cells of the sessions placed there whose clients are still connected
at t, served or waiting -- among the GPUs whose connected footprint plus the new session's fits
the per-GPU budget. If none fits, it goes to the GPU with the smallest connected footprint and
waits in that GPU's queue. Ties go to the lower index. Cells are the measure of load because a
round's time is steps x cells / throughput (the tunnels of a round run concurrently).

``python -m torch.distributed.run --nproc-per-node N wind-tunnel_b200/placement.py`` runs the
config-5 workload over N GPUs: the same Poisson stream as one GPU, each rank serving its share,
a barrier before the window, and rank 0 printing the merged statistics (frame latencies pooled
over every GPU, throughput summed). Ranks exchange only that barrier and the final statistics,
over a CPU (gloo) group.
"""
import argparse
import heapq
import json
import os

import numpy as np

import lbm
import serving


class Placer:
    """Deterministic least-connected-cells placement of sessions on ``gpus`` GPUs, each with
    ``budget_bytes`` of HBM for sessions; ``footprint(session)`` is the bytes a session
    charges. ``place(session, t)`` must be called in arrival order (t non-decreasing)."""

    def __init__(self, gpus, budget_bytes, footprint):
        if gpus < 1:
            raise ValueError('placement needs at least one GPU')
        self.gpus = int(gpus)
        self.budget = int(budget_bytes)
        self.footprint = footprint
        self.cells = [0] * self.gpus       # connected cells per GPU
        self.bytes = [0] * self.gpus       # connected footprint per GPU
        self.placed = [0] * self.gpus      # sessions placed per GPU, all time
        self.placed_cells = [0] * self.gpus
        self.assignment = []               # the GPU of every session placed, in arrival order
        self._ends = []                    # (departure, sequence, session id) of known lifetimes
        self._live = {}                    # session id -> (gpu, cells, bytes) while connected
        self._seq = 0
        self._last_t = float('-inf')

    def _drop(self, sid):
        g, n, b = self._live.pop(sid)
        self.cells[g] -= n
        self.bytes[g] -= b

    def _depart(self, t):
        while self._ends and self._ends[0][0] <= t:
            sid = heapq.heappop(self._ends)[2]
            if sid in self._live:
                self._drop(sid)

    def leave(self, session, t):
        """The session's client disconnected at t (a front end that does not know lifetimes
        reports departures this way; every rank must see the same departures in the same order
        as the arrivals). Unknown or already departed sessions are ignored."""
        t = float(t)
        if t < self._last_t:
            raise ValueError('departures must be reported in time order with the arrivals')
        self._last_t = t
        self._depart(t)
        if session.id in self._live:
            self._drop(session.id)

    def place(self, session, t):
        t = float(t)
        if t < self._last_t:
            raise ValueError('sessions must be placed in arrival order')
        self._last_t = t
        self._depart(t)
        need = int(self.footprint(session))
        fits = [g for g in range(self.gpus) if self.bytes[g] + need <= self.budget]
        if fits:
            g = min(fits, key=lambda g: (self.cells[g], g))
        else:
            g = min(range(self.gpus), key=lambda g: (self.bytes[g], g))
        self.cells[g] += session.n
        self.bytes[g] += need
        self.placed[g] += 1
        self.placed_cells[g] += session.n
        self._live[session.id] = (g, session.n, need)
        if session.lifetime != float('inf'):
            heapq.heappush(self._ends, (t + session.lifetime, self._seq, session.id))
        self._seq += 1
        self.assignment.append(g)
        return g


def merge(stats, latencies):
    """One summary of per-GPU serving statistics: ``stats[r]`` is rank r's ``simulate`` result
    and ``latencies[r]`` its frame latencies in seconds. Latency percentiles are taken over
    every GPU's frames together; counts and throughput are summed."""
    lat = np.concatenate([np.asarray(l, np.float64) for l in latencies]) * 1e3
    if lat.size == 0:
        lat = np.zeros(1)
    total = lambda k: sum(s[k] for s in stats)
    return {'gpus': len(stats), 'frames': int(total('frames')),
            'p50_ms': round(float(np.percentile(lat, 50)), 2), 'p99_ms': round(float(np.percentile(lat, 99)), 2),
            'max_ms': round(float(lat.max()), 2),
            'admitted': int(total('admitted')), 'abandoned': int(total('abandoned')),
            'retired': int(total('retired')), 'failed': int(sum(s.get('failed', 0) for s in stats)),
            'mean_active': round(float(total('mean_active')), 1),
            'glups': round(float(total('glups')), 3),
            'step_glups_device': round(float(total('step_glups_device')), 3),
            'peak_used_gb_max': max(s['peak_used_gb'] for s in stats),
            'per_gpu': [{k: s[k] for k in ('frames', 'p50_ms', 'p99_ms', 'admitted', 'abandoned', 'mean_active',
                                           'glups', 'peak_used_gb', 'placed')} for s in stats]}


def simulate_rank(rank, world, precision='fp32', budget=160e9, particles=5000, barrier=None, placer=None, **kw):
    """This rank's share of ``serving.simulate``: every rank draws the same arrival stream and
    serves the sessions the Placer puts on it. Returns (statistics, frame latencies in s).
    The session footprint is the one admission charges (``lbm.estimate_bytes``)."""
    if placer is None:
        placer = Placer(world, budget, lambda s: lbm.estimate_bytes(s.dims, precision, s.particles))
    lat = []
    out = serving.simulate(precision=precision, budget=budget, particles=particles,
                           keep=lambda s, t: placer.place(s, t) == rank, before_window=barrier,
                           latencies_out=lat, **kw)
    out['placed'] = placer.placed[rank]
    out['placed_all'] = placer.placed[:]
    return out, lat


def main(argv=None):
    import torch
    import torch.distributed as dist
    ap = argparse.ArgumentParser(description='Config-5 serving over the GPUs of one node (one rank per GPU)')
    ap.add_argument('--duration', type=float, default=300.0)
    ap.add_argument('--rate', type=float, default=2.0, help='arrivals per second per GPU')
    ap.add_argument('--mean-life', type=float, default=60.0)
    ap.add_argument('--budget-gb', type=float, default=160.0, help='per GPU')
    ap.add_argument('--precision', nargs='+', default=['fp32', 'fp16'])
    ap.add_argument('--steps-per-frame', type=int, default=10)
    ap.add_argument('--seed', type=int, default=5)
    ap.add_argument('--warmup', type=float, default=3.0, help='untimed seconds of rounds before the window')
    a = ap.parse_args(argv)
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group('gloo', timeout=datetime.timedelta(minutes=10))
    ms = serving.masks()
    for prec in a.precision:
        barrier = dist.barrier if world > 1 else None
        out, lat = simulate_rank(rank, world, precision=prec, budget=a.budget_gb * 1e9, barrier=barrier,
                                 duration=a.duration, rate=a.rate * world, mean_life=a.mean_life, seed=a.seed,
                                 device=f'cuda:{local}', steps_per_frame=a.steps_per_frame, mask_set=ms,
                                 warmup_s=a.warmup)
        if world > 1:
            gathered = [None] * world
            dist.all_gather_object(gathered, (out, lat))
        else:
            gathered = [(out, lat)]
        if rank == 0:
            m = merge([g[0] for g in gathered], [g[1] for g in gathered])
            m.update(precision=prec, duration_s=a.duration, arrival_rate=a.rate * world, mean_lifetime_s=a.mean_life,
                     budget_gb_per_gpu=a.budget_gb)
            print(json.dumps(m), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
