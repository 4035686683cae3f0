"""Replay of the reference server's recorded Engine (tests/golden/engine_trace.npz).

The fixture holds the Solver calls the reference's own Engine made (server/app.py:104-202)
while a scripted client drove it over a real WebSocket, and the frames the server sent. A
replay issues the same calls, in the same order and with the same arguments, on any Solver
with the reference's API, and packs each frame as the Engine packs it (server/app.py:172-194):
header keys in the Engine's order, parts in parts16, parts8, slice, cp order, `steps` the
steps since the last frame or explicit reset. `mlups` is wall-clock time in the recording,
so the replay takes it from the recorded frame.
"""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'engine_trace.npz')


def load():
    """(events with arrays resolved, recorded frame bytes, particle seed)."""
    with np.load(GOLDEN) as z:
        events = json.loads(bytes(z['events']).decode())
        for ev in events:
            for k, v in list(ev.items()):
                if isinstance(v, dict) and set(v) == {'array'}:
                    ev[k] = z[v['array']]
        frames = [z[f'frame_{j}'].tobytes() for j in range(sum(1 for k in z.files if k.startswith('frame_')))]
        seed = int(z['particle_seed'])
    return events, frames, seed


def replay(events, recorded, make_solver):
    """Frames the Engine sends when it drives make_solver(dims)'s Solver with `events`."""
    import wire
    s, steps_since, out, prev = None, 0, [], None
    for ev in events:
        m = ev['method']
        if m == 'init':
            s = make_solver(tuple(ev['dims']))
        elif m == 'reset':
            s.reset(ev['uin'])
            if prev != 'init':  # a client's 'reset' (a new grid's reset keeps the count)
                steps_since = 0
        elif m == 'set_solid':
            s.set_solid(ev['solid'])
        elif m == 'set_surface':
            s.set_surface(ev['verts'], ev['norms'])
        elif m == 'set_particles':
            s.set_particles(ev['count'], ev['p'])
        elif m == 'step':
            s.step(ev['steps'], ev['p'])
            steps_since += ev['steps']
        elif m == 'frame':
            o = s.frame(ev['p'], ev['want_cp'])
            rec = wire.decode(recorded[len(out)])['header']
            header = {'type': 'frame', 'dims': [s.nx, s.ny, s.nz], 'numP': s.num_p, 'numVerts': s.num_verts,
                      'forces': o['forces'], 'steps': steps_since, 'mlups': rec['mlups'],
                      'running': bool(ev['p'].get('running'))}
            parts = [(k, o[k]) for k in ('parts16', 'parts8', 'slice', 'cp') if k in o]
            if 'slice' in o:
                header.update(sliceW=o['sliceW'], sliceH=o['sliceH'], sliceAxis=o['sliceAxis'])
            steps_since = 0
            out.append(wire.pack(header, parts))
        prev = m
    return out
