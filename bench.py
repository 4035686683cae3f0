"""Benchmark of the wind-tunnel LBM hot path on B200.

Workload (default): 512x256x256 = 33.5M cells, FP32 populations, a seeded union of six
axis-aligned ellipsoids (semi-axes 10-60 cells) resting on a moving ground belt,
u = 0.05, nu = 0.001 (tau = 0.503), Smagorinsky Cs = 0.16. One bench step is one frame
of the reference's serving loop: 10 LBM steps, particle advection (2000 streamline
particles seeded on the inlet plane), packing, a 512x256 speed slice at mid-height,
surface pressure on every boundary cell and the momentum-exchange force.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line. `value` is aggregate GLUPS over all ranks with the lattice resident
in HBM; `e2e` is a whole session through the public Solver API (mask and surface upload,
reset, then K frames each with its outputs read back to pinned host memory). Populations
(5.1 GB) are far larger than L2, so no flush is needed between steps.

N > 1 runs independent replicas, one tunnel per GPU ("replicas only": independent
tunnels never exchange data); time is the max over ranks.

The line also carries, for the fp32 default run: `roofline` (the fused step alone against the
HBM peak, with a 2 GiB device copy timed in the same run beside it), `cpu_baseline` (the
oracle on the host cores), `precision_variants` (fp32 fast, fp16 and bf16 shifted storage,
fp16 exact), `accuracy_vs_fp64` (a chaotic and a laminar regime against an fp64 run; with
`--accuracy-long` also the chaotic regime's statistics over 40,000 steps),
`batching` (the 24-tunnel batch of config 4 under both batch executors, every tunnel re-run
alone and compared bit for bit), and `voxelize` (the server-side voxeliser on the benchmark
body). At N = 1 it carries `serving`: the config-5 serving loop (Poisson sessions of
0.5-33.5M cells under a 160 GB budget, 30 frames/s requested per session) run from its
stationary population, after 3 s of untimed rounds, for `--serving` seconds per storage
precision, with p50/p99 frame latency, admitted sessions and aggregate GLUPS.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'wind-tunnel_b200'))

STEPS_PER_FRAME = 10
N_PARTICLES = 2000
ALGO_BYTES = {'fp32': 152, 'fp16': 76, 'bf16': 76, 'fp64': 304}  # per cell per LBM step
METRIC = 'GLUPS & % of HBM roofline, FP16-store vs FP32 at stated error; p99 frame ms'


def env_int(k, d):
    return int(os.environ.get(k, d))


def peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as fh:
            m = json.load(fh)
        return float(m['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def copy_bandwidth(dev, nbytes=2 << 30, reps=5):
    """Device-to-device copy bandwidth on this GPU now (read + write bytes per second, GB/s):
    torch's copy of a buffer 16x larger than L2, best of `reps`, CUDA events."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    dst = torch.empty_like(src)
    src.fill_(1)
    dst.copy_(src)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float('inf')
    for _ in range(reps):
        ev0.record()
        dst.copy_(src)
        ev1.record()
        ev1.synchronize()
        best = min(best, ev0.elapsed_time(ev1) / 1e3)
    del src, dst
    torch.cuda.empty_cache()
    return 2 * nbytes / best / 1e9


def profile_traffic(name):
    """dram bytes per launch from a committed ncu summary (profiles/<name>), if present."""
    path = os.path.join(ROOT, 'profiles', name)
    try:
        for line in open(path):
            if line.startswith('traffic_bytes_per_step:'):
                return float(line.split(':', 1)[1].split()[0])
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    FIELDS = ['clocks.sm', 'clocks.max.sm', 'power.draw', 'utilization.gpu', 'clocks_event_reasons.hw_slowdown',
              'clocks_event_reasons.hw_thermal_slowdown', 'clocks_event_reasons.sw_thermal_slowdown',
              'clocks_event_reasons.sw_power_cap']

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ['nvidia-smi', f'--id={self.gpu}', '--query-gpu=' + ','.join(self.FIELDS),
                 '--format=csv,noheader,nounits', '-lms', '200'],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        """Median SM clock over the samples taken under load (GPU utilization >= 50%), the
        maximum clock and every throttle reason seen active in any sample."""
        sm, loaded, mx, reasons = [], [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) != len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
                if float(parts[3]) >= 50.0:
                    loaded.append(sm[-1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:]):
                if v.lower().startswith('active'):
                    reasons.add(nm)
        if not sm:
            return {'sm_mhz': None, 'sm_max_mhz': None, 'reasons': [], 'samples': 0}
        return {'sm_mhz': statistics.median(loaded or sm), 'sm_max_mhz': mx, 'reasons': sorted(reasons),
                'samples': len(sm), 'samples_under_load': len(loaded)}


def frame_params(dims):
    nx, ny, nz = dims
    return dict(uIn=0.05, tau=3 * 0.001 + 0.5, smag=0.16, steps=STEPS_PER_FRAME,
                maxAge=2.2 * nx / (0.05 * STEPS_PER_FRAME), lref=40.0,
                seedX=2.0, seedCy=(ny - 1) / 2, seedCz=(nz - 1) / 2, seedHy=(ny - 4) / 2, seedHz=(nz - 4) / 2,
                slice=dict(axis=1, index=ny // 2, field=0, vmin=0.0, vmax=1.6), cp=True)


def build_workload(scale):
    import bodies
    dims, solid, p = bodies.config2(scale=scale)
    verts, norms = bodies.surface_points(solid, dims)
    return dims, solid, verts, norms


def step_kernels(tile):
    """The kernels one step of step-tile `tile` launches (the tile table of csrc/wt_kernels.cuh)."""
    if 8 <= tile <= 17:
        return 'k_step_stream + k_step_faces'
    if tile in (27, 28):
        return 'k_step_rows with the face cells fused in'
    if 19 <= tile <= 35 and tile != 29:
        return 'k_step_rows + k_step_faces'
    return 'k_step_bulk + k_step_faces'


STEP_REPEATS, STEP_CHUNK = 5, 50
TUNE_DEVELOP = 1000  # steps of flow development before the autotuner times the tiles


def step_time(solver, p, ev0, ev1):
    """Seconds per LBM step: median of STEP_REPEATS timings of STEP_CHUNK steps each, CUDA
    events on the tunnel's stream (the populations, 2.5-5 GB at 33.5M cells, exceed L2)."""
    import torch
    reps = []
    for _ in range(STEP_REPEATS):
        torch.cuda.synchronize(solver.dev)
        ev0.record(solver.stream)
        solver.step(STEP_CHUNK, p)
        ev1.record(solver.stream)
        ev1.synchronize()
        reps.append(ev0.elapsed_time(ev1) / 1e3 / STEP_CHUNK)
    return statistics.median(reps), reps


def run_ours(args, rank, world, local_rank):
    import torch
    import lbm

    dev = torch.device('cuda', local_rank)
    torch.cuda.set_device(dev)
    dims, solid, verts, norms = build_workload(args.scale)
    nx, ny, nz = dims
    n = nx * ny * nz
    p = frame_params(dims)
    prec = args.precision

    import ranks
    barrier = ranks.barrier

    def max_over_ranks(x):
        return ranks.max_over_ranks(x, dev)

    # ---- device-resident frame loop ----
    s = lbm.Solver(dims, dev, precision=prec, seed=1234 + rank, collision=args.collision)
    s.set_solid(solid)
    s.set_surface(verts, norms)
    s.reset(p['uIn'])
    s.set_particles(N_PARTICLES, p)
    import autotune
    if args.tile:
        tile, tile_ms = args.tile, {}
        s.set_tile(tile)
    else:
        # part of the warm-up, on a developed flow, with the four fastest tiles of the screen run
        # off in sustained windows (short windows under the power cap rank the heavier tiles too
        # high)
        tile, tile_ms = autotune.tune(s, p, force=True, develop=TUNE_DEVELOP, finalists=4)
    launches_per_frame = 2 * STEPS_PER_FRAME + 1 + 1 + 1 + 1 + 2  # steps, advect, pack, slice, cp, forces(2)

    def frame_device():
        s.step(STEPS_PER_FRAME, p)
        s.launch_frame(p, want_cp=True, copy=False)  # outputs stay on the device

    for _ in range(args.warmup):
        frame_device()
    s.synchronize()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the clock sampler runs across every device-timed region below (frames, step, variants)
    clk = ClockSampler(local_rank).__enter__()
    torch.cuda.synchronize(dev)
    ev0.record(s.stream)
    for _ in range(args.steps):
        frame_device()
    ev1.record(s.stream)
    torch.cuda.synchronize(dev)
    barrier()
    t_dev = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    value = ranks.whole_job_rate(n * STEPS_PER_FRAME * args.steps, t_dev) / 1e9

    # ---- LBM step alone: roofline of the fused step (bulk + face kernels) ----
    t_step, step_reps = step_time(s, p, ev0, ev1)
    hbm, peak_kind = peaks()
    achieved = ALGO_BYTES[prec] * n / t_step / 1e9
    copy_here = copy_bandwidth(dev)
    # DRAM bytes per step from the committed capture (a 384x192x192 case scaled to the full grid)
    traffic = profile_traffic(f'step_{prec}_384x192x192.md') if (nx, ny, nz) == (512, 256, 256) else None
    roofline = {'bound': 'hbm', 'achieved': round(achieved, 1), 'peak': hbm, 'unit': 'GB/s',
                'frac': round(achieved / hbm, 4), 'traffic': traffic,
                'peak_source': f'{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)' if peak_kind == 'measured'
                else 'fallback 6.65 TB/s', 'kernel': f'wt_step ({prec}) = {step_kernels(tile)}, one LBM step',
                'algorithmic_bytes_per_cell': ALGO_BYTES[prec], 'step_ms': round(t_step * 1e3, 4),
                'copy_gbs_this_run': round(copy_here, 1), 'frac_of_copy_this_run': round(achieved / copy_here, 4),
                'glups_step_only': round(n / t_step / 1e9, 3), 'tile': tile,
                'timing': f'median of {STEP_REPEATS} repeats of {STEP_CHUNK} steps (CUDA events on the tunnel stream)',
                'step_ms_repeats': [round(x * 1e3, 4) for x in step_reps],
                'tile_ms_per_step': {str(k): round(v, 4) for k, v in tile_ms.items()},
                'tiles_timed': (f'by the autotuner after {TUNE_DEVELOP} steps of flow development: median of 3 '
                                'interleaved 8-step windows per tile, then the 4 fastest in 3 interleaved '
                                '100-step windows') if not args.tile
                               else 'tile given on the command line'}
    del s
    torch.cuda.empty_cache()

    # ---- end to end through the public Solver API, host buffers ----
    host_solid = torch.from_numpy(solid).pin_memory().numpy()
    host_verts = torch.from_numpy(verts).pin_memory().numpy()
    host_norms = torch.from_numpy(norms).pin_memory().numpy()
    frame_ms = []
    barrier()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    s = lbm.Solver(dims, dev, precision=prec, seed=99 + rank, collision=args.collision)
    s.set_tile(tile)
    s.set_solid(host_solid)
    s.set_surface(host_verts, host_norms)
    s.reset(p['uIn'])
    s.set_particles(N_PARTICLES, p)
    d2h = 0
    for _ in range(args.steps):
        tf = time.perf_counter()
        s.step(STEPS_PER_FRAME, p)
        out = s.frame(p, want_cp=True)
        frame_ms.append((time.perf_counter() - tf) * 1e3)
        d2h = sum(out[k].nbytes for k in ('parts16', 'parts8', 'slice', 'cp')) + 6 * 8
    torch.cuda.synchronize(dev)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    h2d_total = solid.nbytes + verts.nbytes + norms.nbytes + N_PARTICLES * 16
    e2e = {'value': round(ranks.whole_job_rate(n * STEPS_PER_FRAME * args.steps, t_e2e) / 1e9, 3), 'unit': 'GLUPS',
           'h2d_bytes_per_step': int(round(h2d_total / args.steps)), 'd2h_bytes_per_step': int(d2h),
           'what': 'one session through lbm.Solver: set_solid + set_surface + reset + set_particles, then K frames of '
                   'step(10) + frame() with outputs copied to pinned host memory',
           'frame_ms': {'p50': round(float(np.percentile(frame_ms, 50)), 3),
                        'p99': round(float(np.percentile(frame_ms, 99)), 3)}}
    del s
    torch.cuda.empty_cache()

    # ---- storage-precision / collision-form variants of the step (same workload) ----
    variants = {}
    if args.variants and prec == 'fp32':
        for vp, vc in (('fp32', 'fast'), ('fp16', 'fast'), ('bf16', 'fast'), ('fp16', 'exact')):
            v = lbm.Solver(dims, dev, precision=vp, collision=vc)
            v.set_solid(solid)
            v.reset(p['uIn'])
            vtile, vms = autotune.tune(v, p, force=True, develop=TUNE_DEVELOP, finalists=4)
            v.step(5, p)
            tv, _ = step_time(v, p, ev0, ev1)
            variants[f'{vp}-{vc}'] = {'glups_step_only': round(n / tv / 1e9, 3),
                            'achieved_gbs': round(ALGO_BYTES[vp] * n / tv / 1e9, 1),
                            'speedup_vs_fp32_step': round(t_step / tv, 3), 'tile': vtile,
                            'tile_ms_per_step': {str(k): round(x, 4) for k, x in vms.items()}}
            del v
            torch.cuda.empty_cache()

    clk.__exit__(None, None, None)

    batching = run_batching(dev) if args.batch and prec == 'fp32' else None
    vox = run_voxelize(dev) if args.batch and prec == 'fp32' else None

    acc = None
    if args.accuracy and prec == 'fp32' and rank == 0:
        import accuracy
        acc = {'chaotic_nu0.001': accuracy.study(steps=args.accuracy_steps, scale=0.5, device=dev),
               'laminar_nu0.02': accuracy.study(steps=2 * args.accuracy_steps, scale=0.5, device=dev, nu=0.02)}
        if args.accuracy_long:
            acc['statistics_nu0.001'] = accuracy.long_study(device=dev)

    return dict(value=value, t_dev=t_dev, roofline=roofline, e2e=e2e, clocks=clk.summary(), accuracy=acc,
                batching=batching, voxelize=vox,
                launches=launches_per_frame * args.steps, dims=dims, n=n, variants=variants)


def run_batching(dev, replays=5, graph_steps=100):
    """Config 4: 24 tunnels (0.5M-8M cells, 2:1:1, own obstacles and flow parameters) in one
    batch: one bulk kernel over every tunnel plus a face kernel per step, captured as a CUDA
    graph of `graph_steps` steps. The batch tile (a persistent work-list loop, one block per
    work-list tile, or the tunnels' descriptors in the kernel parameters) is picked by timing
    each batched tile shape. The streams executor (every tunnel's own kernel on its own stream, forked and
    joined inside one graph) is timed the same way. Every tunnel is then re-run alone for
    every step both executors made and compared bit for bit (populations, mac, forces), with
    its rate alone beside it."""
    import torch
    import bodies
    import lbm
    from batch import TunnelBatch
    cfg = bodies.config4()
    solvers, params = [], []
    for dims, solid, p in cfg:
        s = lbm.Solver(dims, dev)
        s.set_solid(solid)
        s.reset(p['uIn'])
        solvers.append(s)
        params.append(p)
    cells = sum(s.n for s in solvers)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tile_ms, steps_done = {}, 0
    # a persistent form, grid forms (100 + k), then the parameter-space forms (200 + k)
    for tile in (7, 103, 118, 203, 218, 229):
        b = TunnelBatch(solvers, params, tile=tile)
        b.step(2)
        ev0.record(b.stream)
        b.step(4)
        ev1.record(b.stream)
        ev1.synchronize()
        tile_ms[tile] = ev0.elapsed_time(ev1) / 4
        steps_done += 6
        b.close()
    tile = min(tile_ms, key=tile_ms.get)
    b = TunnelBatch(solvers, params, tile=tile)
    b.capture(graph_steps)
    b.replay()
    steps_done += graph_steps
    b.synchronize()
    ev0.record(b.stream)
    for _ in range(replays):
        b.replay()
    ev1.record(b.stream)
    ev1.synchronize()
    steps_done += replays * graph_steps
    t = ev0.elapsed_time(ev1) / 1e3
    b.close()
    # the streams executor: each tunnel's own kernel on its own stream, all at once, the
    # fork and join captured as one graph of the same length
    b = TunnelBatch(solvers, params, mode='streams')
    b.capture(graph_steps)
    b.replay()
    steps_done += graph_steps
    b.synchronize()
    ev0.record(b.stream)
    for _ in range(replays):
        b.replay()
    ev1.record(b.stream)
    ev1.synchronize()
    steps_done += replays * graph_steps
    ts = ev0.elapsed_time(ev1) / 1e3
    b.close()
    # every tunnel re-run alone for the same steps: populations compared bit for bit on the
    # device, forces (fp64, deterministic) exactly, and the tunnel's own rate alone
    per, alone_s = [], 0.0
    for k, (dims, solid, p) in enumerate(cfg):
        alone = lbm.Solver(dims, dev)
        alone.set_solid(solid)
        alone.reset(p['uIn'])
        ev0.record(alone.stream)
        alone.step(steps_done, p)
        ev1.record(alone.stream)
        ev1.synchronize()
        ta = ev0.elapsed_time(ev1) / 1e3
        alone_s += ta
        b_s = solvers[k]
        same = bool(torch.equal(alone.f[alone.cur], b_s.f[b_s.cur]) and torch.equal(alone.mac[alone.cur], b_s.mac[b_s.cur]))
        f_alone, f_batch = alone.forces6(), b_s.forces6()
        per.append({'dims': list(dims), 'cells': alone.n, 'bit_identical': same,
                    'forces_identical': bool(np.array_equal(f_alone, f_batch)),
                    'cd_batch': round(float(f_batch[3] / (0.5 * p['uIn'] ** 2 * max(1, bodies.areas(solid, dims)[0]))), 6),
                    'alone_glups': round(alone.n * steps_done / ta / 1e9, 3)})
        del alone
    torch.cuda.empty_cache()
    out = {'tunnels': len(solvers), 'cells': cells, 'tile': tile,
           'tile_ms_per_step': {str(a): round(v, 3) for a, v in tile_ms.items()},
           'graph_steps': graph_steps, 'replays': replays, 'ms_per_step': round(t / (replays * graph_steps) * 1e3, 4),
           'glups': round(cells * replays * graph_steps / t / 1e9, 3),
           'streams': {'ms_per_step': round(ts / (replays * graph_steps) * 1e3, 4),
                       'glups': round(cells * replays * graph_steps / ts / 1e9, 3)},
           'alone_sequential_glups': round(cells * steps_done / alone_s / 1e9, 3),
           'checked_steps': steps_done, 'tunnels_bit_identical_to_alone': sum(r['bit_identical'] for r in per),
           'per_tunnel': per}
    del solvers
    torch.cuda.empty_cache()
    return out


def run_voxelize(dev, repeats=3):
    """Server-side voxeliser (web/js/voxelize.js on the GPU) on the benchmark body: the six
    ellipsoids of the 512x256x256 workload as triangle meshes, timed end to end (mesh upload,
    all stages, mask and areas back on the host), and compared with the analytic mask of the
    same ellipsoids (they differ only in surface cells)."""
    import bodies
    import voxel
    dims = (512, 256, 256)
    analytic, params = bodies.ellipsoid_union(dims, 6, 2024, scale=1.0, floor='belt')
    tris = np.concatenate([bodies.ellipsoid_mesh((cx, cy, cz), (a, b, c), 48, 96) for cx, cy, cz, a, b, c in params])
    voxel.voxelize(tris, dims, ground=True, device=dev)  # warm-up (module load, allocator)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        solid, st = voxel.voxelize(tris, dims, ground=True, device=dev)
        times.append(time.perf_counter() - t0)
    n = dims[0] * dims[1] * dims[2]
    differ = int((solid != analytic).sum())
    return {'dims': list(dims), 'triangles': int(len(tris)), 'crossings': st['crossings'],
            'ms': round(min(times) * 1e3, 2), 'gcells_per_s': round(n / min(times) / 1e9, 3),
            'solid_cells': st['count'], 'frontal': st['frontal'], 'planform': st['planform'],
            'cells_differing_from_analytic': differ, 'fraction_differing': round(differ / n, 6)}


def cpu_baseline(dims, solid, budget_s, threads=None):
    """The oracle (C++ restatement of the reference kernels, OpenMP) on the host cores:
    whole-grid LBM steps of the same workload until `budget_s` seconds have been spent."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle
    cores = oracle.set_threads(threads or os.cpu_count() or 1)
    L = oracle.Lattice(dims, oracle.F32)
    L.solid[:] = solid
    L.reset(0.05)
    L.step(1, 0.05, 0.503, 0.16)  # warm-up (page faults)
    t0 = time.perf_counter()
    k = 0
    while True:
        L.step(1, 0.05, 0.503, 0.16)
        k += 1
        if time.perf_counter() - t0 > budget_s:
            break
    dt = time.perf_counter() - t0
    n = dims[0] * dims[1] * dims[2]
    return {'value': round(k * n / dt / 1e9, 5), 'unit': 'GLUPS', 'cores': cores, 'kind': 'port',
            'sample': f'{k} whole-grid LBM steps of {dims[0]}x{dims[1]}x{dims[2]} (oracle/lbm_oracle.cpp, '
                      f'OpenMP, {cores} threads); Warp CPU backend unavailable on this box'}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=200)
    ap.add_argument('--warmup', type=int, default=5)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--precision', default='fp32', choices=['fp32', 'fp16', 'bf16', 'fp64'])
    ap.add_argument('--collision', default=None, choices=['exact', 'fast'],
                    help='collision form (default: exact for fp32/fp64, fast for fp16/bf16)')
    ap.add_argument('--tile', type=int, default=0, help='step tile variant (0 = autotune)')
    ap.add_argument('--scale', type=float, default=1.0, help='grid scale (1.0 = 512x256x256)')
    ap.add_argument('--cpu-budget', type=float, default=12.0)
    ap.add_argument('--no-cpu', action='store_true')
    ap.add_argument('--no-variants', dest='variants', action='store_false')
    ap.add_argument('--no-accuracy', dest='accuracy', action='store_false')
    ap.add_argument('--no-batch', dest='batch', action='store_false')
    ap.add_argument('--accuracy-steps', type=int, default=2000)
    ap.add_argument('--accuracy-long', action='store_true',
                    help='add the 40,000-step statistics regime to the accuracy study')
    ap.add_argument('--serving', type=float, default=20.0,
                    help='seconds of the config-5 serving run per precision (0 = skip; N = 1 only)')
    args = ap.parse_args()

    world = env_int('WORLD_SIZE', 1)
    rank = env_int('RANK', 0)
    local_rank = env_int('LOCAL_RANK', 0)

    if args.impl == 'reference':
        return run_reference(args, rank, world)

    import torch
    import torch.distributed as dist
    if world > 1:
        from datetime import timedelta
        dist.init_process_group('nccl', timeout=timedelta(seconds=120),
                                device_id=torch.device('cuda', local_rank))
    r = run_ours(args, rank, world, local_rank)
    serving_out = None
    if world == 1 and args.serving > 0 and args.precision == 'fp32':
        import serving
        ms = serving.masks()
        serving_out = {}
        for prec in ('fp32', 'fp16'):
            serving_out[prec] = serving.simulate(duration=args.serving, precision=prec, device=f'cuda:{local_rank}',
                                                 mask_set=ms, warmup_s=3.0)
            torch.cuda.empty_cache()
    cpu = None
    if rank == 0 and not args.no_cpu:
        import bodies
        dims, solid, _ = bodies.config2(scale=args.scale)
        cpu = cpu_baseline(dims, solid, args.cpu_budget)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    nx, ny, nz = r['dims']
    line = {
        'metric': METRIC, 'value': round(r['value'], 3), 'unit': 'GLUPS', 'n_gpus': world, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': round(r['t_dev'] / args.steps * 1e3, 4), 'higher_is_better': True,
        'scaling': 'weak', 'vs_baseline': None, 'dtype': {'fp32': 'f32', 'fp16': 'f16-store/f32',
                                                          'bf16': 'bf16-store/f32', 'fp64': 'f64'}[args.precision],
        'data': 'synthetic (seeded ellipsoid-union obstacle, PCG64 seed 2024)',
        'config': {'workload': f'{nx}x{ny}x{nz} D3Q19 regularized-LBM + Smagorinsky, {args.precision} populations, '
                               f'6-ellipsoid body on moving belt, frame = {STEPS_PER_FRAME} steps + {N_PARTICLES} '
                               f'particles + {nx}x{nz} slice + surface Cp + forces',
                   'cells': r['n'], 'steps_per_frame': STEPS_PER_FRAME, 'l2': 'inputs larger than L2 (no flush)',
                   'parallelism': f'replicas x{world}'},
        'roofline': r['roofline'], 'cpu_baseline': cpu, 'e2e': r['e2e'], 'clocks': r['clocks'],
        'gpu_launches': r['launches'], 'precision_variants': r['variants'], 'accuracy_vs_fp64': r['accuracy'],
        'batching': r['batching'], 'voxelize': r['voxelize'], 'serving': serving_out,
    }
    print(json.dumps(line), flush=True)


def run_reference(args, rank, world):
    """The reference's CPU implementation of the path timed on the host cores: the oracle
    port (C++ restatement of server/lbm.py's kernels), all threads, one whole-grid LBM step
    per bench step. Rank 0 only."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import bodies
    import oracle
    dims, solid, p = bodies.config2(scale=args.scale)
    cores = oracle.set_threads(os.cpu_count() or 1)
    L = oracle.Lattice(dims, oracle.F32)
    L.solid[:] = solid
    L.reset(p['uIn'])
    for _ in range(args.warmup):
        L.step(1, p['uIn'], p['tau'], p['smag'])
    t0 = time.perf_counter()
    for _ in range(args.steps):
        L.step(1, p['uIn'], p['tau'], p['smag'])
    dt = time.perf_counter() - t0
    n = dims[0] * dims[1] * dims[2]
    v = n * args.steps / dt / 1e9
    nx, ny, nz = dims
    line = {'impl': 'reference', 'metric': METRIC, 'value': round(v, 5), 'unit': 'GLUPS', 'n_gpus': world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': round(dt / args.steps * 1e3, 3),
            'higher_is_better': True, 'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f32',
            'data': 'synthetic (seeded ellipsoid-union obstacle, PCG64 seed 2024)',
            'config': {'workload': f'{nx}x{ny}x{nz} D3Q19 regularized-LBM + Smagorinsky, fp32 populations, '
                                   f'6-ellipsoid body on moving belt', 'cells': n},
            'cpu_baseline': {'value': round(v, 5), 'unit': 'GLUPS', 'cores': cores, 'kind': 'port',
                             'sample': f'1 whole-grid LBM step of {nx}x{ny}x{nz} per bench step (oracle port, '
                                       f'OpenMP {cores} threads); Warp CPU backend unavailable on this box'},
            'e2e': {'value': round(v, 5), 'unit': 'GLUPS', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


if __name__ == '__main__':
    main()
