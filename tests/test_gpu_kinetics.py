"""Kinetic synapse waveforms on the device against the oracle: ExpTwo,
Alpha and ExpThree conductances (P/api/net/network/step.rs:206-398; the
ExpOne profile is covered by the HH tests), each integrated exactly per step
from the arriving jumps, the current g * (E_rev - V) added to the neuron's
input in profile order."""
import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg

pytestmark = pytest.mark.gpu

HH = 4
EXPTWO, ALPHA, EXPTHREE = 1, 2, 3


def _network(make_net, n=300, k=10, steps=3000, seed=9):
    rng = np.random.default_rng(seed)
    dt = 0.01
    net = make_net()
    p = net.add_population(HH, n)
    for col, v in enumerate([dt, 1.0, 120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 0.0, 0.0]):
        net.fill_param(p, col, v)
    net.set_param(p, 8, rng.normal(10.0, 2.0, n).astype(np.float32))
    net.set_state(p, 0, rng.uniform(-70, -60, n).astype(np.float32))
    net.fill_state(p, 1, 0.0529)
    net.fill_state(p, 2, 0.5961)
    net.fill_state(p, 3, 0.3177)
    k2 = net.register_kinetics(EXPTWO, [0.5, 5.0], 0.0, dt)
    ka = net.register_kinetics(ALPHA, [2.0], -80.0, dt)
    k3 = net.register_kinetics(EXPTHREE, [0.3, 3.0, 20.0, 0.7, 0.3], 0.0, dt)
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    post = rng.integers(0, n, pre.size).astype(np.uint32)
    order = np.lexsort((post, pre))
    pre, post = pre[order], post[order]
    st = rng.choice(np.array([k2, ka, k3], np.uint8), pre.size)
    net.connect(p, pre, p, post, rng.uniform(0.0, 0.3, pre.size).astype(np.float32),
                rng.integers(1, 30, pre.size).astype(np.uint8), syn_types=st)
    net.build()
    raster = []
    for _ in range(steps):
        net.step(1)
        raster.append(np.asarray(net.spikes(p)).copy())
    return net, p, np.array(raster)


def test_exptwo_alpha_expthree_bit_identical_to_the_oracle():
    g, gp, rg = _network(lambda: sg.Network(0))
    c, cp, rc = _network(lambda: O.Network(0))
    assert rg.sum() > 500                 # past the onset volley: every neuron fires again
    assert np.array_equal(rg, rc)
    for col in range(4):
        assert np.array_equal(g.state(gp, col).view(np.uint32), c.state(cp, col).view(np.uint32))
    g.close()


def test_kinetics_validated():
    """P/api/net/synapse.rs:95-158 and its tests :310-340."""
    net = sg.Network(0)
    net.add_population(HH, 4)
    for kind, params in ((EXPTWO, [3.0, 1.0]), (EXPTWO, [2.0, 2.0]), (EXPTWO, [0.0, 3.0]), (ALPHA, [0.0]),
                         (EXPTHREE, [1.0, 0.5, 3.0, 1.0, 1.0]), (EXPTHREE, [0.5, 1.0, 3.0, 0.0, 0.0]),
                         (EXPTHREE, [0.5, 1.0, 3.0, -1.0, 1.0]), (7, [1.0])):
        with pytest.raises(sg.SimuseError):
            net.register_kinetics(kind, params, 0.0, 0.01)
    net.close()
