"""Wire format of the WebSocket frames, pinned to frames written by the reference's own
``pack`` (server/app.py:23-41; fixtures from tests/golden/make_golden.py --frames)."""
import json
import struct

import numpy as np
import pytest

import wire
from conftest import golden

FR = golden('frames.npz')
CASES = range(int(FR['cases']))


def _case(k):
    header = json.loads(FR[f'header_{k}'].tobytes().decode())
    names = [str(n) for n in FR[f'names_{k}'] if str(n)]
    return header, [(n, FR[f'{n}_{k}']) for n in names], FR[f'frame_{k}'].tobytes()


@pytest.mark.parametrize('k', CASES)
def test_pack_matches_reference_bytes(k):
    header, parts, ref = _case(k)
    assert wire.pack(header, parts) == ref


@pytest.mark.parametrize('k', CASES)
def test_decode_round_trip(k):
    header, parts, ref = _case(k)
    d = wire.decode(ref)
    h = dict(d['header'])
    h.pop('offsets')
    assert h == header
    assert (4 + struct.unpack_from('<I', ref)[0]) % 8 == 0  # payload 8-byte aligned
    for name, arr in parts:
        np.testing.assert_array_equal(d[name], arr.view(wire.PART_DTYPE[name]))
    assert set(wire.PART_ORDER) & set(d) == {n for n, _ in parts}


@pytest.mark.parametrize('k', CASES)
def test_layout_frame_equals_pack(k):
    """A payload assembled at FrameLayout offsets (as the device does) gives the same bytes."""
    header, parts, ref = _case(k)
    p = dict(parts)
    num_p = len(p['parts8']) if 'parts8' in p else 0
    wh = (header['sliceW'], header['sliceH']) if 'slice' in p else None
    nv = len(p['cp']) if 'cp' in p else 0
    lay = wire.FrameLayout(num_p, wh, nv)
    buf = np.zeros(lay.total_bytes, np.uint8)
    for name, arr in parts:
        raw = np.ascontiguousarray(arr).view(np.uint8)
        assert raw.size == lay.sizes[name]
        buf[lay.offsets[name]:lay.offsets[name] + raw.size] = raw
    assert lay.forces_offset % 8 == 0 and lay.total_bytes == lay.payload_bytes + 48
    assert lay.frame(header, buf) == ref


# ---- client uploads (web/js/net.js:9-16, 85-92 framing; server/app.py:138-148, 218-222 checks) ----
def test_upload_framing_round_trip():
    import gzip
    import struct
    header = {'type': 'solid', 'dims': [4, 3, 3]}
    body = bytes(range(36))
    msg = wire.encode_upload(header, body)
    hl = struct.unpack_from('<I', msg, 0)[0]
    assert msg[4:4 + hl].decode() == '{"type":"solid","dims":[4,3,3]}'
    h, payload = wire.decode_upload(msg)
    assert h == header and gzip.decompress(payload) == body


def test_upload_arrays_accepts_what_the_engine_accepts():
    mask = (np.arange(36) % 3).astype(np.uint8)
    h, p = wire.decode_upload(wire.encode_upload({'type': 'solid', 'dims': [4, 3, 3]}, mask.tobytes()))
    kind, arr = wire.upload_arrays(h, p, (4, 3, 3))
    assert kind == 'solid' and np.array_equal(arr, mask)
    vn = np.arange(2 * 6, dtype=np.float32)
    h, p = wire.decode_upload(wire.encode_upload({'type': 'surface', 'numVerts': 2}, vn.tobytes()))
    kind, verts, norms = wire.upload_arrays(h, p, (4, 3, 3))
    assert kind == 'surface'
    assert np.array_equal(verts, vn[:6].reshape(2, 3)) and np.array_equal(norms, vn[6:].reshape(2, 3))


def test_upload_arrays_ignores_what_the_engine_ignores():
    mask = np.zeros(36, np.uint8)
    for header, body, dims in [({'type': 'solid', 'dims': [4, 3, 4]}, mask, (4, 3, 3)),        # another grid
                               ({'type': 'solid', 'dims': [4, 3, 3]}, mask[:35], (4, 3, 3)),   # short mask
                               ({'type': 'surface', 'numVerts': 3}, np.zeros(12, np.float32), (4, 3, 3)),
                               ({'type': 'unknown'}, mask, (4, 3, 3))]:
        h, p = wire.decode_upload(wire.encode_upload(header, body.tobytes()))
        assert wire.upload_arrays(h, p, dims) is None
