"""Record the reference server driving a Solver over a real WebSocket.

Runs the reference's own ``server/app.py`` of RICKxxROLLING/wind-tunnel: its Engine thread,
its ``ws_handler`` and its ``pack()``, imported read-only from the reference checkout. Its
``warp`` calls (``app.py:12, 56-59, 114, 151, 249``: import, device query, synchronize,
set_device, init) are answered by a stand-in module, and its ``lbm`` module is the reference's
own ``server/lbm.py`` (loaded under the same stand-in, as oracle/warp_shim.py does) with
``Solver`` replaced by ``oracle/engine_solver.OracleSolver``: the reference Solver's API
computed by the oracle, which equals the reference kernels bit for bit.

A scripted client then speaks the browser's protocol (web/js/net.js) over ``/ws``: it asks for
the 'test' resolution, waits for the first frame, uploads a gzip mask and a gzip surface in the
binary message format, sets parameters, asks for particles, and acknowledges frames with
``ready``, changing parameters and resetting the flow along the way. Written to
``engine_trace.npz`` beside this script:

* ``events``: the Engine's Solver calls in order (JSON: method and arguments; arrays by key),
  up to and including the call that made the last frame the client took;
* ``frame_<j>``: the bytes of each binary frame the server sent;
* ``hello``: the server's greeting; ``particle_seed``: the seed of set_particles' generator.

tests/test_engine_trace.py replays the calls on the oracle and checks the frames come back;
tests/test_gpu_engine_trace.py replays them on the library's CUDA Solver.

    python tests/golden/make_engine_trace.py <reference root>    (or set WT_REFERENCE_ROOT)
"""
import asyncio
import importlib.util
import json
import os
import sys
import threading
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, 'oracle'), os.path.join(ROOT, 'wind-tunnel_b200'), HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

NFRAMES = 8
RES = 'test'


def warp_stand_in():
    """The shim's warp module plus the runtime calls the server makes."""
    import warp_shim
    wp = warp_shim.make_stub(np.float32)

    class Device:
        is_cuda = True
        name = 'oracle (CPU stand-in for the GPU)'
        total_memory = 16 << 30

    wp.get_preferred_device = lambda: Device()
    wp.synchronize = lambda: None
    wp.set_device = lambda d: None
    wp.init = lambda: None
    return wp


def load_reference_server(ref):
    """The reference's server/app.py with its lbm.Solver replaced by OracleSolver."""
    from engine_solver import OracleSolver
    sys.modules['warp'] = warp_stand_in()
    spec = importlib.util.spec_from_file_location('lbm', os.path.join(ref, 'server', 'lbm.py'))
    lbm = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(lbm)
    lbm.Solver = OracleSolver
    sys.modules['lbm'] = lbm
    spec = importlib.util.spec_from_file_location('reference_app', os.path.join(ref, 'server', 'app.py'))
    app = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(app)
    return app


def client_script(dims):
    """The client's messages: uploads and parameters after the first frame, then changes."""
    import bodies
    import wire
    solid, _ = bodies.ellipsoid_union(dims, 3, 811, scale=dims[0] / 256.0, floor='belt')
    verts, norms = bodies.surface_points(solid, dims)
    surf = np.concatenate([verts.reshape(-1), norms.reshape(-1)]).astype(np.float32).tobytes()
    nx, ny, nz = dims
    setup = [wire.encode_upload({'type': 'solid', 'dims': list(dims)}, solid.tobytes()),
             wire.encode_upload({'type': 'surface', 'numVerts': len(verts)}, surf),
             {'type': 'params', 'uIn': 0.07, 'tau': 0.515, 'particles': 400, 'maxAge': 300.0,
              'seedCy': (ny - 1) / 2, 'seedCz': (nz - 1) / 2, 'seedHy': ny / 4, 'seedHz': nz / 4,
              'slice': {'axis': 2, 'index': nz // 2, 'field': 0, 'vmin': 0.0, 'vmax': 1.5}, 'cp': True},
             {'type': 'respawn'}]
    later = {3: [{'type': 'params', 'steps': 7, 'smag': 0.18,
                  'slice': {'axis': 1, 'index': ny // 3, 'field': 2, 'vmin': 0.0, 'vmax': 2.0}}],
             5: [{'type': 'reset'}],
             6: [{'type': 'params', 'running': False}]}
    return setup, later


async def run_client(port, dims):
    import aiohttp
    from aiohttp import WSMsgType
    setup, later = client_script(dims)
    frames, hello = [], None
    async with aiohttp.ClientSession() as cs:
        async with cs.ws_connect(f'http://127.0.0.1:{port}/ws', max_msg_size=1 << 30) as ws:
            hello = await ws.receive_json(timeout=60)
            await ws.send_json({'type': 'grid', 'res': RES})
            while (await ws.receive_json(timeout=120))['type'] != 'grid':
                pass
            while len(frames) < NFRAMES:
                msg = await ws.receive(timeout=120)
                if msg.type == WSMsgType.TEXT:
                    continue
                frames.append(bytes(msg.data))
                if len(frames) == NFRAMES:
                    break  # no 'ready': the server sends nothing more
                for m in (setup if len(frames) == 1 else later.get(len(frames), [])):
                    if isinstance(m, dict):
                        await ws.send_json(m)
                    else:
                        await ws.send_bytes(m)
                await ws.send_json({'type': 'ready'})
    return hello, frames


def record(ref):
    from aiohttp import web
    app_mod = load_reference_server(ref)
    from engine_solver import OracleSolver
    box, ready = {}, threading.Event()

    def serve():
        loop = asyncio.new_event_loop()
        asyncio.set_event_loop(loop)
        app = web.Application()
        app.on_startup.append(app_mod.on_startup)
        app.router.add_get('/ws', app_mod.ws_handler)
        runner = web.AppRunner(app)
        loop.run_until_complete(runner.setup())
        site = web.TCPSite(runner, '127.0.0.1', 0)
        loop.run_until_complete(site.start())
        box.update(port=runner.addresses[0][1], loop=loop)
        ready.set()
        loop.run_forever()

    threading.Thread(target=serve, daemon=True).start()
    ready.wait(60)
    dims = app_mod.RESOLUTIONS[RES]
    hello, frames = asyncio.run(run_client(box['port'], dims))
    time.sleep(0.2)
    trace = list(OracleSolver.instances[-1].trace)
    # up to the call that made the client's last frame
    k = [i for i, (m, _) in enumerate(trace) if m == 'frame'][len(frames) - 1]
    return hello, frames, trace[:k + 1]


def save(hello, frames, trace):
    arrays, events = {}, []
    for i, (method, args) in enumerate(trace):
        ev = {'method': method}
        for name, v in args.items():
            if isinstance(v, np.ndarray):
                key = f'a{i}_{name}'
                arrays[key] = v
                ev[name] = {'array': key}
            else:
                ev[name] = v
        events.append(ev)
    out = {f'frame_{j}': np.frombuffer(f, np.uint8) for j, f in enumerate(frames)}
    out.update(arrays)
    out['events'] = np.frombuffer(json.dumps(events).encode(), np.uint8)
    out['hello'] = np.frombuffer(json.dumps(hello).encode(), np.uint8)
    from engine_solver import OracleSolver
    out['particle_seed'] = np.array(OracleSolver.seed_for_particles)
    np.savez_compressed(os.path.join(HERE, 'engine_trace.npz'), **out)


def main():
    from make_golden import reference_root
    ref = reference_root(sys.argv)
    hello, frames, trace = record(ref)
    save(hello, frames, trace)
    print(f'{len(frames)} frames, {len(trace)} Solver calls '
          f'({", ".join(sorted({m for m, _ in trace}))})')


if __name__ == '__main__':
    main()
