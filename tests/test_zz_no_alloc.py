"""wt_forces_noalloc: the force reduction for callers that cannot allocate device memory.

Those callers (a host framework that owns the GPU's memory pool and lends this library only
its inputs and outputs, or a per-frame loop where an allocation would synchronise the device)
get block partials from an array built into libwt.so instead of caller scratch. This test
calls the entry point through the C ABI on two calls in a row and checks each against
wt_forces, which uses caller-provided scratch, to fp64 rounding: the two partition the link
list into blocks differently, so each component may differ by rounding of the order of 1e-16
times the sum of the magnitudes it adds up, which for a component that nearly cancels can be
far above 1e-12 of the component itself. The tolerance is therefore relative 1e-12 plus an
absolute 1e-12 of the largest component. It also checks that a list longer than the built-in limit is refused before
any launch. Run alone in a fresh process, its first call performs the per-device set-up.
"""
import numpy as np
import pytest
import torch

import wtlib as W

pytestmark = pytest.mark.gpu


def test_forces_noalloc_matches_forces_on_consecutive_calls():
    import bodies
    from lbm import Solver
    dims = (96, 40, 40)
    solid = bodies.sphere_tunnel(dims, (30, 20, 20), 9.0, floor='noslip')
    s = Solver(dims, 'cuda:0')
    s.set_solid(solid)
    s.reset(0.05)
    assert s.n_links > 256  # several reduction blocks
    p = dict(uIn=0.05, tau=0.506, smag=0.16)
    out = torch.empty(6, dtype=torch.float64, device='cuda:0')
    for _ in range(2):
        s.step(15, p)
        ref = s.forces6()  # wt_forces with caller scratch
        out.fill_(float('nan'))
        torch.cuda.synchronize()
        W.call('wt_forces_noalloc', s.gp, s.cur, W.ptr(s.link_cells), W.ptr(s.link_masks), s.n_links, W.ptr(out), s.sh)
        s.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got))
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * float(np.abs(ref).max()))


def test_forces_noalloc_refuses_lists_beyond_its_limit():
    import bodies
    from lbm import Solver
    dims = (32, 16, 16)
    s = Solver(dims, 'cuda:0')
    s.set_solid(bodies.sphere_tunnel(dims, (10, 8, 8), 3.0))
    out = torch.zeros(6, dtype=torch.float64, device='cuda:0')
    rc = W.lib().wt_forces_noalloc(s.gp, 0, W.ptr(s.link_cells), W.ptr(s.link_masks), W.NOALLOC_MAX_LINKS + 1,
                                   W.ptr(out), s.sh)
    assert rc == W.WT_ERR_CAPACITY
    assert b'limit' in W.lib().wt_last_error()
