"""The serving arena's ranges (host logic; no GPU): first fit at 256-byte alignment, merging of
freed neighbours, and a random sequence of allocations and releases checked against a
byte-occupancy model."""
import random

import arena


def test_first_fit_alignment_and_merge():
    a = arena.Arena(10 * 256)
    x = a.alloc(100)    # rounds up to 256
    y = a.alloc(512)
    z = a.alloc(256)
    assert (x, y, z) == (0, 256, 768) and a.free == [(1024, 1536)]
    assert a.alloc(2000) is None and a.largest() == 1536
    a.release(y)
    assert a.free == [(256, 512), (1024, 1536)]
    assert a.alloc(300) == 256  # the first range that fits, not the largest
    a.release(256)
    a.release(x)                # merges with the range after it
    assert a.free == [(0, 768), (1024, 1536)]
    a.release(z)                # merges both sides: one range again
    assert a.free == [(0, 2560)] and not a.used and a.free_bytes() == a.size


def test_random_sequence_matches_an_occupancy_model():
    rng = random.Random(7)
    a = arena.Arena(64 * 1024)
    occ = bytearray(a.size)
    live = []
    for _ in range(1500):
        if live and (rng.random() < 0.45 or len(live) > 40):
            off = live.pop(rng.randrange(len(live)))
            n = a.used[off]
            assert all(occ[off:off + n])
            occ[off:off + n] = bytes(n)
            a.release(off)
        else:
            n = rng.randrange(1, 6000)
            off = a.alloc(n)
            need = (n + 255) // 256 * 256
            # first fit: no earlier free run of `need` bytes at a 256-byte boundary exists
            first = next((o for o in range(0, a.size - need + 1, 256) if not any(occ[o:o + need])), None)
            assert off == first
            if off is not None:
                assert off % 256 == 0 and not any(occ[off:off + need])
                occ[off:off + need] = b'\x01' * need
                live.append(off)
        # the free list is exactly the unoccupied bytes, merged and sorted
        runs, o = [], 0
        while o < a.size:
            if occ[o]:
                o += 1
                continue
            e = o
            while e < a.size and not occ[e]:
                e += 1
            runs.append((o, e - o))
            o = e
        assert a.free == runs
