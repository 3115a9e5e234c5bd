"""The c3 ensemble definition on the CPU: seeded, inside the stated ranges, and sized for one B200."""
import numpy as np

from si3d_b200 import ensemble, replicas


def test_draw_is_seeded_and_in_range():
    a = ensemble.basins(n=8, seed=5)
    b = ensemble.basins(n=8, seed=5)
    for x, y in zip(a, b):
        assert (x.nx, x.ny, x.nlayers) == (y.nx, y.ny, y.nlayers)
        np.testing.assert_array_equal(x.depth, y.depth)
        np.testing.assert_array_equal(x.uair, y.uair)
    for m in a:
        assert 200 <= m.nx <= 1000 and 100 <= m.ny <= 800 and 20 <= m.nlayers <= 60
        wet = m.depth > 0
        assert 0.6 < wet.mean() < 0.8
        assert m.depth[wet].min() >= 2.0 and m.depth.max() <= m.nlayers
        tau = m.seeds["stress_mean"]
        assert 0.05 <= tau <= 0.2


def test_full_draw_fits_one_gpu_and_splits_evenly():
    ms = ensemble.basins()
    assert len(ms) == 64
    total = sum(ensemble.device_bytes(m) for m in ms)
    assert total < 170e9
    parts = replicas.partition([ensemble.device_bytes(m) for m in ms], 8)
    assert replicas.imbalance([ensemble.device_bytes(m) for m in ms], parts) < 1.1
