"""Dopamine-modulated eligibility learning on the device against the oracle.

The device keeps the reference's lazy Brain (P/api/learn/brain.rs) bound to
the network: per-neuron traces in the neuron kernel, one eligibility kernel
per step over the synapses of spiking neurons, rewards folding every
eligibility to now before the weight update.  Every FP32 operation is the
oracle's, so traces, eligibility, weights and the rasters that follow from
the changed weights must be the oracle's bits.
"""
import numpy as np
import pytest

import oracle as O
import scenarios as S
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

CFG = dict(dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=0.5, w_min=0.0, w_max=4.0)


def _same(a, b):
    return np.array_equal(np.asarray(a, np.float32).view(np.uint32), np.asarray(b, np.float32).view(np.uint32))


def _scripted(make_net, n=24, steps=600):
    pre, post, w = S.lcg_net(0xC0FFEE, n)
    rng = np.random.default_rng(1)
    spikes = (rng.random((steps, n)) < 0.18).astype(np.int32)
    acts = {}
    for t in range(steps):
        a = []
        if t == 5:
            a.append(("snapshot", ()))
        if t % 12 == 7:
            a += [("reward", (1.2,)), ("learning_state", ()), ("weights", ())]
        if t % 50 == 20:
            a += [("reward", (-0.7, 0.4)), ("weights", ())]
        if t % 97 == 30:
            a += [("reward", (3.0, 1.0, 64.0)), ("weights", ())]
        if t == 250:
            a += [("clear_eligibility", ()), ("learning_state", ())]
        if t == 300:
            a += [("restrict_eligibility", (np.arange(pre.size) % 3 != 0,)), ("learning_state", ())]
        if t == 350:
            a += [("set_eligibility", (np.linspace(-1.0, 1.0, pre.size, dtype=np.float32),)), ("learning_state", ())]
        if t == 400:
            a += [("recall", (0.25,)), ("weights", ())]
        if t % 100 == 99:
            a.append(("motor_counts", ()))
        if a:
            acts[t] = a
    net, out = S.learn_scripted(make_net, n, pre, post, w, spikes, CFG, acts, motor=((0, 8), (8, 24)))
    return net, out


def test_scripted_learning_bit_identical_to_the_oracle():
    g, og = _scripted(lambda: sg.Network(0))
    c, oc = _scripted(lambda: O.Network(0))
    assert len(og) == len(oc) > 50
    for (t, verb, rg), (_, _, rc) in zip(og, oc):
        if verb == "learning_state":
            for a, b in zip(rg[:3], rc[:3]):
                assert _same(a, b), (t, verb)
            assert rg[3] == rc[3] == t + 1
        elif verb == "weights":
            assert _same(rg, rc), (t, verb)
        else:
            assert rg == rc, (t, verb)
    assert _same(g.weights(), c.weights())
    g.close()


def _driven(make_net, steps=600, reward_every=50):
    """The balanced LIF network with Poisson drive (exact-sum rings before
    learning), learning on from step 0 with rewards of alternating sign."""
    net = make_net()
    spec = W.lif_balanced(n=2000, k_in=100, seed=3, ext_rate_hz=4000.0, ext_weight=100.0, w_exc=20.0, g=5.0)
    p = W.build_lif(net, spec, device_generator=isinstance(net, sg.Network))
    net.build()
    net.enable_learning(dt=0.1, tau_pre=20.0, tau_post=20.0, tau_e=200.0, a_ltp=0.1, a_ltd=0.12, lr=2.0,
                        w_min=-150.0, w_max=60.0)
    w0 = net.weights()
    raster, states = [], []
    for t in range(steps):
        net.step(1)
        raster.append(np.asarray(net.spikes(p)).copy())
        if t % reward_every == reward_every - 1:
            net.reward(1.0 if (t // reward_every) % 2 == 0 else -0.5)
            states.append(net.learning_state())
    return net, p, np.array(raster), states, w0


def test_driven_network_learning_bit_identical_to_the_oracle():
    g, gp, rg, sg_, w0 = _driven(lambda: sg.Network(0))
    assert g.scatter_mode == "ordered"      # rewards change weights: the ordered path
    c, cp, rc, sc, _ = _driven(lambda: O.Network(0))
    assert rg.sum() > 1000
    assert np.array_equal(rg, rc)
    for a, b in zip(sg_, sc):
        for x, y in zip(a[:3], b[:3]):
            assert _same(x, y)
        assert a[3] == b[3]
    wg, wc = g.weights(), c.weights()
    assert _same(wg, wc)
    assert np.count_nonzero(wg != w0) > 1000          # rewards moved many weights
    assert _same(g.state(gp, 0), c.state(cp, 0))
    assert _same(g.ring(0), c.ring(0))
    g.close()


def test_learning_errors():
    net = sg.Network(0)
    p = net.add_population(S.LIF, 8)
    net.connect(p, np.arange(7, dtype=np.uint32), p, np.arange(1, 8, dtype=np.uint32), np.ones(7, np.float32),
                np.ones(7, np.uint8))
    with pytest.raises(sg.SimuseError):     # not built
        net.enable_learning()
    net.build()
    with pytest.raises(sg.SimuseError):     # not enabled
        net.reward(1.0)
    with pytest.raises(sg.SimuseError):
        net.enable_learning(tau_e=0.0)
    net.enable_learning()
    with pytest.raises(sg.SimuseError):     # twice
        net.enable_learning()
    with pytest.raises(sg.SimuseError):     # ceiling below the floor
        net.reward(1.0, 1.0, -1.0)
    with pytest.raises(sg.SimuseError):
        net.restrict_eligibility(np.ones(3, np.uint8))
    with pytest.raises(sg.SimuseError):
        net.set_eligibility(np.ones(3, np.float32))
    net.close()
    b = sg.Network(0)
    q = b.add_population(S.LIF, 8)
    b.connect(q, np.arange(7, dtype=np.uint32), q, np.arange(1, 8, dtype=np.uint32), np.ones(7, np.float32),
              np.ones(7, np.uint8))
    b.set_weight_format(sg.W_BF16)
    b.build()
    with pytest.raises(sg.SimuseError):     # BF16 weights are read-only
        b.enable_learning()
    b.close()


def test_per_network_reward_in_a_pool_bit_identical_to_the_oracle():
    """Three networks pooled as populations of one device network, each
    rewarded on its own synapse range (the oracle's pooled reward equals
    each network alone, tests/test_oracle_learn.py)."""
    steps = 300
    cr = S.pool_creatures(steps)
    g, _, gr = S.learn_pool(lambda: sg.Network(0), cr, CFG, steps)
    c, _, cr_ = S.learn_pool(lambda: O.Network(0), cr, CFG, steps)
    assert gr == cr_
    assert _same(g.weights(), c.weights())
    for a, b in zip(g.learning_state()[:3], c.learning_state()[:3]):
        assert _same(a, b)
    with pytest.raises(sg.SimuseError):
        g.reward(1.0, synapses=(0, g.num_synapses + 1))
    g.close()
