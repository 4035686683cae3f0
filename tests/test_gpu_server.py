"""The WebSocket front end (server.py) driven over real sockets by two scripted browser clients.

Each client speaks the reference protocol as the browser does (web/js/net.js): it reads the
`hello`, asks for a resolution with `grid`, and after the first frame uploads a gzip mask and a
gzip surface in the binary message format, sets parameters, asks for particles (`respawn`),
changes parameters again mid-run, and acknowledges every frame with `ready`. The two clients
run at once on different grids, so their sessions step together in the server's rounds. Every
frame each client receives is decoded (wire.decode, the client's decodeFrame) and must equal,
byte for byte, the frame the same session gives when its tunnel runs alone with the same
commands applied the reference Engine's way (server/app.py:104-193) before the same frames.
"""
import asyncio
import json
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NFRAMES = 7


def _start(srv):
    """Serve `srv` through server.make_app on 127.0.0.1 (an ephemeral port) in a thread."""
    from aiohttp import web
    import server
    box, ready = {}, threading.Event()

    def main():
        loop = asyncio.new_event_loop()
        asyncio.set_event_loop(loop)
        app = server.make_app(srv, 'test GPU')
        runner = web.AppRunner(app)
        loop.run_until_complete(runner.setup())
        site = web.TCPSite(runner, '127.0.0.1', 0)
        loop.run_until_complete(site.start())
        box.update(port=runner.addresses[0][1], app=app, loop=loop)
        ready.set()
        loop.run_forever()
        loop.run_until_complete(runner.cleanup())
        loop.close()

    t = threading.Thread(target=main, daemon=True)
    t.start()
    assert ready.wait(60)

    def stop():
        box['loop'].call_soon_threadsafe(box['loop'].stop)
        t.join(60)
    return box, stop


def _script(k, dims):
    """Client k's uploads and parameter messages."""
    import bodies
    import wire
    solid, _ = bodies.ellipsoid_union(dims, 2 + k, 710 + k, scale=dims[0] / 256.0, floor='belt')
    verts, norms = bodies.surface_points(solid, dims)
    surf = np.concatenate([verts.reshape(-1), norms.reshape(-1)]).astype(np.float32).tobytes()
    nx, ny, nz = dims
    setup = [wire.encode_upload({'type': 'solid', 'dims': list(dims)}, solid.tobytes()),
             wire.encode_upload({'type': 'surface', 'numVerts': len(verts)}, surf),
             {'type': 'params', 'uIn': 0.06 + 0.01 * k, 'tau': 0.51 + 0.01 * k, 'particles': 300 + 100 * k,
              'seedCy': (ny - 1) / 2, 'seedCz': (nz - 1) / 2, 'seedHy': ny / 4, 'seedHz': nz / 4,
              'slice': {'axis': 2 - k, 'index': (nz if k == 0 else ny) // 2, 'field': k, 'vmin': 0.0, 'vmax': 1.5},
              'cp': True},
             {'type': 'respawn'}]
    later = {3: [{'type': 'params', 'steps': 6 + k, 'smag': 0.18}], 5: [{'type': 'reset'}]}
    return setup, later


async def _client(port, k, res, dims):
    import aiohttp
    from aiohttp import WSMsgType
    import wire
    setup, later = _script(k, dims)
    frames = []
    async with aiohttp.ClientSession() as cs:
        async with cs.ws_connect(f'http://127.0.0.1:{port}/ws', max_msg_size=1 << 30) as ws:
            hello = await ws.receive_json(timeout=60)
            assert hello['type'] == 'hello' and any(r['name'] == res and r['fits'] for r in hello['resolutions'])
            await ws.send_json({'type': 'grid', 'res': res})
            while True:
                m = await ws.receive_json(timeout=60)
                assert m['type'] != 'error', m
                if m['type'] == 'grid':
                    assert m['dims'] == list(dims)
                    break
            while len(frames) < NFRAMES:
                msg = await ws.receive(timeout=120)
                if msg.type == WSMsgType.TEXT:
                    raise AssertionError(f'client {k}: {msg.data}')
                assert msg.type == WSMsgType.BINARY, msg
                frames.append(bytes(msg.data))
                d = wire.decode(msg.data)  # the browser's decodeFrame must read it
                assert d['header']['type'] == 'frame' and d['header']['dims'] == list(dims)
                n = len(frames)
                for m in (setup if n == 1 else later.get(n, [])):
                    if isinstance(m, dict):
                        await ws.send_json(m)
                    else:
                        await ws.send_bytes(m)
                await ws.send_json({'type': 'ready'})
    return k, frames


def test_two_clients_over_websockets_match_their_sessions_alone():
    import lbm
    import serving
    import server
    from test_gpu_serving import _engine_replay
    specs = [(0, 'test'), (1, 'low')]
    srv = serving.SessionServer('cuda:0', budget_bytes=8e9, precision='fp32', pacing='client', keep_frames=True,
                                rate_in_header=False)
    box, stop = _start(srv)
    try:
        async def both():
            return await asyncio.gather(*[_client(box['port'], k, res, lbm.RESOLUTIONS[res]) for k, res in specs])
        got = dict(asyncio.run(both()))
        fe = box['app']['frontend']
        sessions = {tuple(s.dims): s for s in fe.sessions.values()}
    finally:
        stop()
    assert not srv.errors, srv.errors
    for k, res in specs:
        dims = lbm.RESOLUTIONS[res]
        s = sessions[tuple(dims)]
        # the commands as the session applied them: (frames before, message, payload)
        script = {}
        for before, msg, payload in s.applied:
            if msg['type'] != 'ready':
                script.setdefault((before, s.id), []).append((msg, payload))
        s0 = serving.Session(s.id, dims, np.zeros(int(np.prod(dims)), np.uint8), dict(server.ENGINE_PARAMS),
                             float('inf'), particles=0, frontal=1)
        s0.p['particles'] = server.ENGINE_PARAMS['particles']
        want = _engine_replay(s0, script, 'fp32', srv.steps_each, NFRAMES)
        assert len(got[k]) == NFRAMES
        for j, (a, b) in enumerate(zip(got[k], want)):
            assert a == b, f'client {k} frame {j} differs from its session run alone'
        hdr = json.loads(got[k][-1][4:4 + int.from_bytes(got[k][-1][:4], 'little')])
        assert hdr['numP'] == 300 + 100 * k and 'slice' in hdr['offsets']
