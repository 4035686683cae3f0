"""Tile autotuner for the fused step kernel.

The step kernel is compiled in several tile shapes (cells per thread along x, threads per
block, minimum resident blocks per SM, which bounds registers); ``wt_step_tiles`` lists
them. All shapes compute bit-identical results. ``tune()`` times each admissible shape
on a tunnel with CUDA events on the tunnel's stream and keeps the fastest; results are
cached per (GPU, precision, grid) in memory and, when ``WT_TILE_CACHE`` names a file,
in that JSON file.

Timing advances the tunnel by ``develop + len(tiles) * (warm + (warm + steps) * repeats)`` LBM
steps (plus ``finalists * (warm + final_steps) * final_repeats``), so tune as a warm-up or on
a scratch tunnel.
"""
import json
import os

import torch

import wtlib as W

_cache = {}
SMEM_LIMIT = 227 * 1024  # dynamic shared memory per block on sm_100


def _key(solver):
    name = torch.cuda.get_device_name(solver.dev)
    return f'{name}|{solver.precision}|{solver.nx}x{solver.ny}x{solver.nz}'


def _load_file():
    path = os.environ.get('WT_TILE_CACHE')
    if path and os.path.exists(path):
        try:
            with open(path) as fh:
                _cache.update(json.load(fh))
        except (OSError, ValueError):
            pass


def _save_file():
    path = os.environ.get('WT_TILE_CACHE')
    if path:
        tmp = path + '.tmp'
        with open(tmp, 'w') as fh:
            json.dump(_cache, fh, indent=1, sort_keys=True)
        os.replace(tmp, path)


def admissible(solver):
    """Tiles the library accepts for this grid: direct-load tiles need nx divisible by their
    cells per thread; streaming tiles (negative second field) need nx divisible by 16."""
    out = []
    elem = {W.F32: 4, W.F16: 2, W.BF16: 2, W.F64: 8}[solver.precision]
    for t in W.step_tiles(solver.precision, solver.collision):
        v = t[1]
        if v > 0 and (solver.nx % v or (solver.precision == W.F64 and v == 4)):
            continue
        if v < 0:
            chunk, stages = -v, t[3]
            smem = stages * (19 * (chunk + 16 // elem) * elem + chunk) + 16 * stages
            if solver.nx % 16 or smem > SMEM_LIMIT:
                continue
        out.append(t)
    return out


def cached(solver):
    _load_file()
    hit = _cache.get(_key(solver))
    return hit['tile'] if hit else None


def _interleaved(solver, params, tiles, steps, warm, repeats, ev0, ev1):
    """Median ms per step of each tile over `repeats` windows of `steps` steps, the windows of
    all tiles interleaved (all tiles once, then all again)."""
    import statistics
    got = {t: [] for t in tiles}
    for _ in range(repeats):
        for t in tiles:
            solver.set_tile(t)
            solver.step(warm, params)
            ev0.record(solver.stream)
            solver.step(steps, params)
            ev1.record(solver.stream)
            ev1.synchronize()
            got[t].append(ev0.elapsed_time(ev1) / steps)
    return {t: statistics.median(v) for t, v in got.items()}


def tune(solver, params, steps=8, warm=2, repeats=3, force=False, develop=0, finalists=0, final_steps=100,
         final_repeats=3):
    """Pick the fastest tile for `solver` and set it; returns (tile, {tile: ms_per_step}).

    Every admissible tile is timed `repeats` times in windows of `steps` steps, the windows
    interleaved across the tiles, and ranked by its median. With `finalists`, the fastest few
    then run off in longer interleaved windows (`final_steps`), and their entries in the returned
    timings are those sustained figures. Under the GPU's power cap, short windows among lighter
    tiles run at higher clocks than the same tile running on its own, and on this workload
    that ranks a tile with more instructions per cell (one-dimensional tile 18) ahead of one
    that is faster in sustained running (row tile 34). `develop` steps (with the current tile)
    come first, so the tiles are timed on a developed flow."""
    if not force:
        hit = cached(solver)
        if hit is not None:
            solver.set_tile(hit)
            return hit, _cache[_key(solver)]['ms']
    if develop:
        solver.step(develop, params)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    tiles = []
    for tile in admissible(solver):
        solver.set_tile(tile[0])
        try:
            solver.step(warm, params)
        except W.WtError:  # e.g. a streaming tile whose stages exceed shared memory
            continue
        tiles.append(tile[0])
    timings = _interleaved(solver, params, tiles, steps, warm, repeats, ev0, ev1)
    if finalists and len(tiles) > 1:
        best = sorted(timings, key=timings.get)[:finalists]
        timings.update(_interleaved(solver, params, best, final_steps, warm, final_repeats, ev0, ev1))
        tid = min(best, key=timings.get)
    else:
        tid = min(timings, key=timings.get)
    solver.set_tile(tid)
    _cache[_key(solver)] = {'tile': tid, 'ms': timings}
    _save_file()
    return tid, timings


def compare(solver, params, tiles, steps=50, repeats=5, developed=1000):
    """Median ms per step of each tile in `tiles`, timed in interleaved repeats (tile order
    inside each repeat) so that clock and power drift fall alike on every tile: first right
    after the caller's reset ('fresh'), then after `developed` more steps with the first tile
    ('developed'). Returns {'fresh': {tile: ms}, 'developed': {tile: ms}}."""
    import statistics
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    out = {}
    for phase in ('fresh', 'developed'):
        if phase == 'developed':
            solver.set_tile(tiles[0])
            solver.step(developed, params)
        reps = {t: [] for t in tiles}
        for _ in range(repeats):
            for t in tiles:
                solver.set_tile(t)
                solver.step(2, params)
                ev0.record(solver.stream)
                solver.step(steps, params)
                ev1.record(solver.stream)
                ev1.synchronize()
                reps[t].append(ev0.elapsed_time(ev1) / steps)
        out[phase] = {t: statistics.median(v) for t, v in reps.items()}
    return out


def main(argv=None):
    """python wind-tunnel_b200/autotune.py [--scale S] FORM:TILE,TILE ... -- compare tiles of each
    storage form (e.g. fp16-fast:21,31) on the benchmark body, fresh and developed."""
    import argparse
    import bodies
    import lbm
    ap = argparse.ArgumentParser(description='compare step tiles on the benchmark body')
    ap.add_argument('forms', nargs='+', help='precision-collision:tile,tile,...')
    ap.add_argument('--scale', type=float, default=1.0, help='grid scale (1.0 = 512x256x256)')
    ap.add_argument('--steps', type=int, default=50)
    ap.add_argument('--repeats', type=int, default=5)
    ap.add_argument('--developed', type=int, default=1000)
    a = ap.parse_args(argv)
    dims, solid, p = bodies.config2(scale=a.scale)
    n = dims[0] * dims[1] * dims[2]
    result = {}
    for spec in a.forms:
        form, tl = spec.split(':')
        prec, coll = form.split('-')
        tiles = [int(t) for t in tl.split(',')]
        s = lbm.Solver(dims, 'cuda:0', precision=prec, collision=coll)
        s.set_solid(solid)
        s.reset(p['uIn'])
        r = compare(s, p, tiles, a.steps, a.repeats, a.developed)
        for phase, ms in r.items():
            for t, v in ms.items():
                print(f'{form} {phase} tile {t}: {v:.4f} ms {n / v / 1e6:.2f} GLUPS', flush=True)
        result[form] = {ph: {str(t): round(v, 4) for t, v in ms.items()} for ph, ms in r.items()}
        del s
        torch.cuda.empty_cache()
    print(json.dumps({'dims': list(dims), 'steps': a.steps, 'repeats': a.repeats, 'developed': a.developed,
                      'ms_per_step': result}))


if __name__ == '__main__':
    main()
