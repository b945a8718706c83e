"""HH + pair STDP over more than one simulated second against the oracle.

HH is chaotic: one flipped bit in a membrane potential eventually moves a
spike.  The device and the oracle share every FP32 operation (RK4 with the
same exponential, no contraction, the reference's ring order, per-edge STDP
updates), so the rasters are expected to stay identical; the test reports
the first step where they differ, if any, and requires it to lie beyond
1 s (100,000 steps of 0.01 ms).
"""
import numpy as np
import pytest

import oracle as O
import scenarios as S
import simuse_b200 as sg

pytestmark = pytest.mark.gpu

STEPS = 110_000      # 1.1 s at dt = 0.01 ms
ONE_SECOND = 100_000


def test_hh_stdp_rasters_match_the_oracle_beyond_one_second():
    g, gpops, _ = S.hh_network(lambda: sg.Network(0), n=500, k_out=12, steps=0)
    c, cpops, _ = S.hh_network(lambda: O.Network(0), n=500, k_out=12, steps=0)
    g.enable_raster(STEPS)
    g.step(STEPS)
    rg = g.read_raster()
    rc = c.step(STEPS, record=True)
    assert rg.shape == rc.shape == (STEPS, 500)
    assert rg.sum() > 10_000                       # the network keeps firing
    diff = np.nonzero((rg != rc).any(axis=1))[0]
    first = int(diff[0]) if diff.size else None
    print(f"HH+STDP 500 neurons: {int(rg.sum())} spikes in {STEPS} steps; first divergent step: {first}")
    assert first is None or first > ONE_SECOND
    if first is None:
        for pg, pc in zip(gpops, cpops):
            assert np.array_equal(g.state(pg, 0).view(np.uint32), c.state(pc, 0).view(np.uint32))
    g.close()
