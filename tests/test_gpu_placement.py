"""Session placement through real tunnels on one GPU: the shares of two ranks are run one
after the other (they never wait on each other), each serving the sessions the shared rule
puts on it. Both runs compute the same assignment, and every session a rank was given is
admitted, abandoned or still queued there."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_two_rank_shares_of_one_stream():
    import lbm
    import placement
    import serving
    masks = {size: [(np.zeros(int(np.prod(dims)), np.uint8), 100.0)] for size, dims in serving.SIZES.items()}
    runs = []
    for rank in range(2):
        placer = placement.Placer(2, 40e9, lambda s: lbm.estimate_bytes(s.dims, 'fp16', s.particles))
        out, lat = placement.simulate_rank(rank, 2, precision='fp16', budget=40e9, particles=500, placer=placer,
                                           duration=1.5, rate=4.0, mean_life=1.0, seed=11, device='cuda:0',
                                           mask_set=masks)
        runs.append((out, lat, placer.assignment))
    common = min(len(r[2]) for r in runs)
    assert common >= 4
    assert runs[0][2][:common] == runs[1][2][:common]
    for rank, (out, lat, assign) in enumerate(runs):
        assert out['frames'] == len(lat) > 0
        assert out['placed'] == assign.count(rank)
        assert out['admitted'] + out['abandoned'] + out['queued_end'] == out['placed']
    m = placement.merge([r[0] for r in runs], [r[1] for r in runs])
    assert m['frames'] == sum(len(r[1]) for r in runs)
    assert m['glups'] > 0
