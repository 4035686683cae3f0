"""WebSocket front end: the reference's `/ws` protocol served by a SessionServer.

The reference server (server/app.py:205-255) accepts browser viewers on `/ws`, greets each with
a `hello` listing the resolutions that fit (server/app.py:77-82), forwards their JSON and binary
messages to one Engine thread through a queue (server/app.py:206-226) and sends back binary
frames and JSON `grid` / `error` messages. This front end speaks the same protocol, message
for message, to the same browser client (web/js/net.js):

* client to server: JSON `grid` {res}, `params`, `respawn`, `reset`, `ready`; binary
  `[u32 header length][JSON {type: 'solid', dims} | {type: 'surface', numVerts}][gzip payload]`;
* server to client: JSON `hello`, `grid` {res, dims}, `error` {message}; binary frames in the
  reference's layout (wire.py), sent once the previous frame was acknowledged with `ready`.

What differs is behind the protocol. The reference runs one tunnel for every client; here each
connection is its own session of a SessionServer (serving.py) on this GPU, admitted against the
HBM budget and stepped with every other session in the same rounds. A `grid` request queues a
session of that resolution (a tunnel of zeros at rest until the client uploads its mask, as the
reference's fresh Solver is); asking for another resolution ends the old session and queues a
new one. The reply `grid` comes at once; a session that then cannot be created gets the
reference's `Could not allocate` error. A closed connection ends its session.

    python wind-tunnel_b200/server.py [--port 8765] [--precision fp32] [--budget-gb 160]
"""
import argparse
import asyncio
import json
import struct
import threading
import time

from aiohttp import WSMsgType, web

import lbm
import serving

# the Engine's parameter dict before a client sets any (server/app.py:61-63)
ENGINE_PARAMS = dict(uIn=0.1, tau=0.51, smag=0.16, steps=10, maxAge=1000.0, lref=40.0, seedX=2.0, seedCy=20.0,
                     seedCz=20.0, seedHy=10.0, seedHz=10.0, slice=None, cp=False, running=True, particles=5000)


class Frontend:
    """The `/ws` endpoint and the serving thread that runs a SessionServer's rounds and sends
    each round's frames and errors to their clients."""

    def __init__(self, srv, loop, gpu_name='CUDA device', memory=None, idle_s=0.002):
        self.srv = srv
        self.loop = loop
        self.gpu_name = gpu_name
        self.memory = memory if memory is not None else int(srv.budget)
        self.idle_s = idle_s
        self.clients = {}          # session id -> WebSocketResponse
        self.sessions = {}         # session id -> Session, every session opened
        self.next_id = 0
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._serve, name='serving', daemon=True)

    # ---- protocol ----
    def hello(self, res=None):
        """The reference's hello (server/app.py:77-82), with fits() answered by admission."""
        table = [{'name': k, 'dims': list(v), 'fits': self.srv.fits(v)} for k, v in lbm.RESOLUTIONS.items()]
        default = 'high' if self.srv.fits(lbm.RESOLUTIONS['high']) else 'test'
        return {'type': 'hello', 'gpu': self.gpu_name, 'cuda': True, 'memory': self.memory, 'resolutions': table,
                'default': default, 'res': res}

    def _send(self, ws, obj):
        coro = ws.send_json(obj) if isinstance(obj, dict) else ws.send_bytes(obj)

        async def go():
            try:
                await coro
            except Exception:  # the client went away; its handler disconnects the session
                pass
        asyncio.run_coroutine_threadsafe(go(), self.loop)

    async def ws_handler(self, request):
        ws = web.WebSocketResponse(max_msg_size=1024 ** 3, heartbeat=20)
        await ws.prepare(request)
        sid, res = None, None
        await ws.send_json(self.hello())
        try:
            async for msg in ws:
                if msg.type == WSMsgType.TEXT:
                    data = json.loads(msg.data)
                    t = data.get('type')
                    if t == 'grid':
                        want = data.get('res')
                        dims = lbm.RESOLUTIONS.get(want)
                        if not dims or not self.srv.fits(dims):
                            await ws.send_json({'type': 'error',
                                                'message': f'Resolution {want} does not fit on this device'})
                            continue
                        if want != res or sid is None:
                            if sid is not None:
                                self.srv.disconnect(sid)
                                self.clients.pop(sid, None)
                            sid, res = self._open(dims), want
                            self.clients[sid] = ws
                        await ws.send_json({'type': 'grid', 'res': res, 'dims': list(dims)})
                    elif sid is not None:
                        self.srv.command(sid, data)
                elif msg.type == WSMsgType.BINARY and sid is not None:
                    buf = msg.data
                    hl = struct.unpack_from('<I', buf, 0)[0]
                    self.srv.command(sid, json.loads(buf[4:4 + hl]), buf[4 + hl:])
        finally:
            if sid is not None:
                self.clients.pop(sid, None)
                self.srv.disconnect(sid)
        return ws

    def _open(self, dims):
        """A new session of this grid: mask of zeros, the Engine's parameters, no particles until
        the client asks for them ('respawn', server/app.py:132-133), no end but its client's."""
        import numpy as np
        sid = self.next_id
        self.next_id += 1
        nx, ny, nz = dims
        s = serving.Session(sid, dims, np.zeros(nx * ny * nz, np.uint8), dict(ENGINE_PARAMS), float('inf'),
                            particles=0, frontal=1)
        s.p['particles'] = ENGINE_PARAMS['particles']
        s.arrival = self.srv.clock()
        self.sessions[sid] = s
        self.srv.enqueue(s)
        return sid

    # ---- serving thread ----
    def _serve(self):
        while not self._stop.is_set():
            n = self.srv.round()
            for sid, frame in self.srv.round_frames:
                ws = self.clients.get(sid)
                if ws is not None:
                    self._send(ws, frame)
            while self.srv.errors:
                sid, message = self.srv.errors.pop(0)
                ws = self.clients.get(sid)
                if ws is not None:
                    self._send(ws, {'type': 'error', 'message': message})
            if n == 0:
                time.sleep(self.idle_s)

    def start(self):
        self._thread.start()

    def stop(self):
        self._stop.set()
        self._thread.join(timeout=10)
        self.srv.close()


def make_app(srv, gpu_name='CUDA device', memory=None):
    """The aiohttp application: `/ws` served by a Frontend over `srv` (started with the app,
    stopped with it)."""
    app = web.Application()
    holder = {}

    async def on_startup(app):
        fe = Frontend(srv, asyncio.get_running_loop(), gpu_name, memory)
        holder['fe'] = fe
        app['frontend'] = fe
        fe.start()

    async def on_cleanup(app):
        holder['fe'].stop()

    async def ws(request):
        return await holder['fe'].ws_handler(request)

    app.on_startup.append(on_startup)
    app.on_cleanup.append(on_cleanup)
    app.router.add_get('/ws', ws)
    return app


def main(argv=None):
    ap = argparse.ArgumentParser(description='WebSocket front end of the wind-tunnel sessions on one GPU')
    ap.add_argument('--port', type=int, default=8765)
    ap.add_argument('--host', default='0.0.0.0')
    ap.add_argument('--precision', default='fp32', choices=['fp32', 'fp16', 'bf16'])
    ap.add_argument('--budget-gb', type=float, default=160.0)
    ap.add_argument('--device', default='cuda:0')
    a = ap.parse_args(argv)
    import torch
    srv = serving.SessionServer(a.device, budget_bytes=a.budget_gb * 1e9, precision=a.precision, pacing='client',
                                admit_thread=True, new_per_round=1)
    name = torch.cuda.get_device_name(torch.device(a.device))
    web.run_app(make_app(srv, name, int(a.budget_gb * 1e9)), host=a.host, port=a.port, print=None)


if __name__ == '__main__':
    main()
