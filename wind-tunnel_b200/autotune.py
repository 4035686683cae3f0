"""Tile autotuner for the fused step kernel.

The step kernel is compiled in several tile shapes (cells per thread along x, threads per
block, minimum resident blocks per SM, which bounds registers); ``wt_step_tiles`` lists
them. All shapes compute bit-identical results. ``tune()`` times each admissible shape
on a tunnel with CUDA events on the tunnel's stream and keeps the fastest; results are
cached per (GPU, precision, grid) in memory and, when ``WT_TILE_CACHE`` names a file,
in that JSON file.

Timing advances the tunnel by ``len(tiles) * (warm + steps) * repeats`` LBM steps, so tune
right after reset (as a warm-up) or on a scratch tunnel.
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


def tune(solver, params, steps=8, warm=2, repeats=2, force=False):
    """Pick the fastest tile for `solver` and set it; returns (tile, {tile: ms_per_step})."""
    if not force:
        hit = cached(solver)
        if hit is not None:
            solver.set_tile(hit)
            return hit, _cache[_key(solver)]['ms']
    timings = {}
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    for tile in admissible(solver):
        tid = tile[0]
        solver.set_tile(tid)
        best = None
        try:
            solver.step(warm, params)
        except W.WtError:  # e.g. a streaming tile whose stages exceed shared memory
            continue
        for _ in range(repeats):
            solver.step(warm, params)
            ev0.record(solver.stream)
            solver.step(steps, params)
            ev1.record(solver.stream)
            ev1.synchronize()
            ms = ev0.elapsed_time(ev1) / steps
            best = ms if best is None else min(best, ms)
        timings[tid] = best
    tid = min(timings, key=timings.get)
    solver.set_tile(tid)
    _cache[_key(solver)] = {'tile': tid, 'ms': timings}
    _save_file()
    return tid, timings
