"""Tsodyks-Markram short-term plasticity on the device against the oracle.

A synapse with a profile delivers weight * R * U with the pre-spike resource
R and release probability U, then depletes R and (facilitating profiles)
raises U; R and U relax toward 1 and U0 between spikes by exact per-step
factors raised to the number of elapsed steps (P/api/net/push.rs:25-102).
The oracle is pinned to the reference's NEURON goldens
(tests/test_oracle_golden.py); here the device must give the oracle's bits.
"""
import numpy as np
import pytest

import oracle as O
import scenarios as S
import simuse_b200 as sg

pytestmark = pytest.mark.gpu

LIF = 1


def test_depressing_synapse_silences_its_post_like_the_oracle():
    g, gs, gp = S.tm_drive(lambda: sg.Network(0))
    c, cs, cp = S.tm_drive(lambda: O.Network(0))
    assert gs > 20 and gp == 0           # P/api/net/network/tests.rs:530-575
    assert (gs, gp) == (cs, cp)
    assert np.array_equal(g.state(0, 0).view(np.uint32), c.state(0, 0).view(np.uint32))
    g.close()


def _mixed(make_net, n=400, k=30, steps=400, seed=4):
    """LIF network with static, depressing and facilitating synapses, delays
    1-10, random input current every step."""
    rng = np.random.default_rng(seed)
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 2.0]):
        net.fill_param(p, col, v)
    net.set_state(p, 0, rng.uniform(-70.0, -55.0, n).astype(np.float32))
    dep = net.register_plasticity(0.5, 100.0, 0.5)
    fac = net.register_plasticity(0.1, 1e6, 0.5, tau_fac=50.0)
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    post = rng.integers(0, n, pre.size).astype(np.uint32)
    order = np.lexsort((post, pre))
    pre, post = pre[order], post[order]
    w = rng.uniform(0.0, 40.0, pre.size).astype(np.float32)
    d = rng.integers(1, 11, pre.size).astype(np.uint8)
    pt = rng.choice(np.array([0, dep, fac], np.uint8), pre.size)
    net.connect(p, pre, p, post, w, d, plast_types=pt)
    net.build()
    idx = np.arange(n, dtype=np.uint32)
    raster = []
    for t in range(steps):
        net.inject_current(p, idx, rng.uniform(0.0, 60.0, n).astype(np.float32))
        net.step(1)
        raster.append(np.asarray(net.spikes(p)).copy())
    return net, p, np.array(raster)


def test_mixed_plastic_network_bit_identical_to_the_oracle():
    g, gp, rg = _mixed(lambda: sg.Network(0))
    c, cp, rc = _mixed(lambda: O.Network(0))
    assert g.scatter_mode == "ordered"
    assert rg.sum() > 1000
    assert np.array_equal(rg, rc)
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert np.array_equal(g.ring(0).view(np.uint32), c.ring(0).view(np.uint32))
    g.close()


def test_plasticity_profiles_validated():
    net = sg.Network(0)
    p = net.add_population(LIF, 4)
    for u0, tau in ((0.0, 1.0), (1.5, 1.0), (0.5, 0.0), (0.5, float("nan"))):
        with pytest.raises(sg.SimuseError):
            net.register_plasticity(u0, tau, 0.5)
    with pytest.raises(sg.SimuseError):
        net.register_plasticity(0.5, 10.0, 0.5, tau_fac=0.0)
    for _ in range(8):
        net.register_plasticity(0.5, 10.0, 0.5)
    with pytest.raises(sg.SimuseError):   # the device holds 8 profiles
        net.register_plasticity(0.5, 10.0, 0.5)
    with pytest.raises(sg.SimuseError):   # profile 9 was not registered
        net.connect(p, np.array([0], np.uint32), p, np.array([1], np.uint32), np.array([1.0], np.float32),
                    np.array([1], np.uint8), plast_types=np.array([9], np.uint8))
    net.close()


def _source_plastic(make_net, n=300, steps=500, seed=8):
    """Poisson sources whose synapses carry Tsodyks-Markram profiles
    (P/api/net/network/step.rs:166-180): each of 40 sources drives 25 random
    posts through static, depressing or facilitating synapses with delays
    0-6, beside recurrent static synapses; some neurons get a plain one-to-one
    drive too."""
    rng = np.random.default_rng(seed)
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 2.0]):
        net.fill_param(p, col, v)
    net.set_state(p, 0, rng.uniform(-70.0, -58.0, n).astype(np.float32))
    dep = net.register_plasticity(0.5, 100.0, 0.5)
    fac = net.register_plasticity(0.1, 1e6, 0.5, tau_fac=50.0)
    for s in range(40):
        src = net.add_poisson_source(300.0 + 20.0 * s, 0.5, 1000 + s)
        posts = rng.choice(n, 25, replace=False).astype(np.uint32)
        w = rng.uniform(5.0, 60.0, 25).astype(np.float32)
        d = rng.integers(0, 7, 25).astype(np.uint8)
        pt = rng.choice(np.array([0, dep, fac], np.uint8), 25)
        net.connect_poisson_source(src, p, posts, w, d, plast_types=pt)
    first = net.add_poisson_sources(n // 2, 200.0, 0.5, seed0=77)
    net.connect_poisson_one_to_one(first, n // 2, p, 12.5, 1)
    pre = np.repeat(np.arange(n, dtype=np.uint32), 10)
    post = rng.integers(0, n, pre.size).astype(np.uint32)
    order = np.lexsort((post, pre))
    net.connect(p, pre[order], p, post[order], rng.uniform(0.0, 20.0, pre.size).astype(np.float32),
                rng.integers(1, 6, pre.size).astype(np.uint8))
    net.build()
    raster = []
    for t in range(steps):
        net.step(1)
        raster.append(np.asarray(net.spikes(p)).copy())
    return net, p, np.array(raster)


def test_plastic_poisson_source_synapses_bit_identical_to_the_oracle():
    g, gp, rg = _source_plastic(lambda: sg.Network(0))
    c, cp, rc = _source_plastic(lambda: O.Network(0))
    assert g.scatter_mode == "ordered"
    assert rg.sum() > 200
    assert np.array_equal(rg, rc)
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert g.events_total == c.events
    g.close()
