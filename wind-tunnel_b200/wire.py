"""Binary frame format of the wind-tunnel WebSocket protocol.

A frame is ``[u32 little-endian header length][JSON header][payload]``. The JSON header is
padded with spaces so the payload starts 8-byte aligned. Its ``offsets`` object gives each
part's byte offset in the payload, and parts start on 8-byte boundaries. The parts are, in
order: ``parts16`` (u16 x 4 per particle), ``parts8`` (u8 per particle), ``slice``
(u8 x 2 per pixel) and ``cp`` (i8 per surface vertex). This is the format the reference
server writes (server/app.py:23-41) and its browser client decodes (web/js/net.js:18-29).

``FrameLayout`` fixes the payload offsets of a tunnel's frame ahead of time. The frame
kernels then write straight into one device buffer at those offsets, and a frame needs one
device-to-host copy (``lbm.Solver.launch_frame_packed``).
"""
import json
import struct

import numpy as np

PART_ORDER = ('parts16', 'parts8', 'slice', 'cp')
PART_DTYPE = {'parts16': np.uint16, 'parts8': np.uint8, 'slice': np.uint8, 'cp': np.int8}


def _align8(n):
    return (n + 7) // 8 * 8


def header_bytes(header, offsets):
    """JSON header with its offsets, space-padded so that 4 + len is a multiple of 8."""
    text = json.dumps(dict(header, offsets=offsets)).encode()
    return text + b' ' * ((8 - (4 + len(text)) % 8) % 8)


def pack(header, parts):
    """Frame bytes for `parts` = [(name, ndarray), ...] in send order."""
    offsets, size = {}, 0
    for name, arr in parts:
        offsets[name] = size
        size = _align8(size + arr.nbytes)
    hb = header_bytes(header, offsets)
    out = bytearray(4 + len(hb) + size)
    out[0:4] = struct.pack('<I', len(hb))
    out[4:4 + len(hb)] = hb
    base = 4 + len(hb)
    for name, arr in parts:
        o = base + offsets[name]
        out[o:o + arr.nbytes] = np.ascontiguousarray(arr).tobytes()
    return bytes(out)


def decode(buf):
    """The browser client's decodeFrame (web/js/net.js:18-29): header dict plus typed views."""
    buf = bytes(buf)
    hl = struct.unpack_from('<I', buf, 0)[0]
    h = json.loads(buf[4:4 + hl].decode())
    base = 4 + hl
    o = h['offsets']
    d = {'header': h}
    counts = {'parts16': lambda: h['numP'] * 4, 'parts8': lambda: h['numP'],
              'slice': lambda: h['sliceW'] * h['sliceH'] * 2, 'cp': lambda: h['numVerts']}
    for name in PART_ORDER:
        if name in o:
            dt = np.dtype(PART_DTYPE[name])
            d[name] = np.frombuffer(buf, dt, counts[name](), base + o[name])
    return d


class FrameLayout:
    """Payload offsets of one tunnel's frame, plus a 48-byte tail that holds the six fp64
    force components (not sent; the host copies them into the header)."""

    def __init__(self, num_p, slice_wh=None, num_verts=0):
        sizes = []
        if num_p:
            sizes += [('parts16', 8 * num_p), ('parts8', num_p)]
        if slice_wh:
            sizes.append(('slice', 2 * slice_wh[0] * slice_wh[1]))
        if num_verts:
            sizes.append(('cp', num_verts))
        self.offsets, self.sizes, pos = {}, {}, 0
        for name, nbytes in sizes:
            self.offsets[name] = pos
            self.sizes[name] = nbytes
            pos = _align8(pos + nbytes)
        self.payload_bytes = pos
        self.forces_offset = pos
        self.total_bytes = pos + 48

    def frame(self, header, payload):
        """Frame bytes from a payload buffer laid out by this layout."""
        hb = header_bytes(header, self.offsets)
        return struct.pack('<I', len(hb)) + hb + bytes(memoryview(payload)[:self.payload_bytes])


# ---- client to server: geometry uploads (web/js/net.js:9-16, 85-92; server/app.py:218-222) ----
def encode_upload(header, payload):
    """A client's binary message: [u32 LE header length][JSON header][gzip of payload], as
    the browser's frameBytes(header, await gzip(bytes)) builds it."""
    import gzip
    hb = json.dumps(header, separators=(',', ':')).encode()  # JSON.stringify's compact form
    return struct.pack('<I', len(hb)) + hb + gzip.compress(bytes(payload))


def decode_upload(buf):
    """(header dict, compressed payload bytes) of a client's binary message, split as the
    reference's WebSocket handler splits it (server/app.py:218-222)."""
    buf = bytes(buf)
    hl = struct.unpack_from('<I', buf, 0)[0]
    return json.loads(buf[4:4 + hl]), buf[4 + hl:]


def upload_arrays(header, payload, dims):
    """The arrays an upload carries, checked as Engine.handle checks them (server/app.py:
    138-148): ('solid', u8[n]) for a mask of exactly this grid, ('surface', verts, norms) for
    numVerts vertices and normals, or None for anything the reference ignores (another grid's
    mask, a size mismatch, an unknown type)."""
    import gzip
    t = header.get('type')
    nx, ny, nz = dims
    if t == 'solid':
        if tuple(header.get('dims', ())) != (nx, ny, nz):
            return None
        arr = np.frombuffer(gzip.decompress(payload), dtype=np.uint8)
        return ('solid', arr) if arr.size == nx * ny * nz else None
    if t == 'surface':
        raw = np.frombuffer(gzip.decompress(payload), dtype=np.float32)
        nv = int(header['numVerts'])
        if raw.size != nv * 6:
            return None
        return 'surface', raw[:nv * 3].reshape(-1, 3), raw[nv * 3:].reshape(-1, 3)
    return None
