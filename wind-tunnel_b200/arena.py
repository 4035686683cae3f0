"""One block of device memory from which serving's tunnels take their per-cell state.

A SessionServer admits tunnels of a few sizes against an HBM budget, and they come and go
every second. Left to torch's caching allocator, tunnels of different sizes fragment its
cache, and an allocation that finds no fitting block makes the allocator free its cache
(synchronising the device) and call cudaMalloc. Under a nearly full budget that took 400-600
ms of a serving round. The arena is allocated once, and tunnels take ranges of it by first
fit at 256-byte alignment; freed ranges merge with free neighbours. No CUDA allocation or free
happens per tunnel.

``Arena(nbytes)`` keeps only the ranges (host logic, testable without a GPU);
``Arena(nbytes, device)`` also holds the device buffer, and ``view(offset, nbytes)`` returns
the uint8 tensor of a range.
"""
import bisect

ALIGN = 256


def _round(n):
    return (int(n) + ALIGN - 1) // ALIGN * ALIGN


class Arena:
    def __init__(self, nbytes, device=None):
        self.size = int(nbytes) // ALIGN * ALIGN  # never more than was asked for
        self.free = [(0, self.size)]  # sorted, disjoint, never adjacent (merged)
        self.used = {}                # offset -> bytes of every range handed out
        self.buf = None
        if device is not None:
            import torch
            self.buf = torch.empty(self.size, dtype=torch.uint8, device=device)

    def largest(self):
        """Bytes of the largest free range."""
        return max((n for _, n in self.free), default=0)

    def free_bytes(self):
        return sum(n for _, n in self.free)

    def alloc(self, nbytes):
        """Offset of a range of `nbytes` (rounded up to 256), the first free one that fits, or
        None."""
        need = _round(nbytes)
        for k, (off, n) in enumerate(self.free):
            if n >= need:
                if n == need:
                    del self.free[k]
                else:
                    self.free[k] = (off + need, n - need)
                self.used[off] = need
                return off
        return None

    def release(self, off):
        """Give a range back; it merges with the free ranges next to it."""
        n = self.used.pop(off)
        k = bisect.bisect_left(self.free, (off, 0))
        if k < len(self.free) and self.free[k][0] == off + n:  # merge with the next
            n += self.free[k][1]
            del self.free[k]
        if k > 0 and self.free[k - 1][0] + self.free[k - 1][1] == off:  # and with the previous
            off, n = self.free[k - 1][0], self.free[k - 1][1] + n
            del self.free[k - 1]
            k -= 1
        self.free.insert(k, (off, n))

    def view(self, off, nbytes):
        """The uint8 device tensor of a range."""
        return self.buf[off:off + _round(nbytes)]
