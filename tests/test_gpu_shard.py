"""A network split across GPUs gives the unsplit network's bits.

The ranks of a split network are emulated in one process on one GPU: each
rank's network keeps its own neurons and the synapses onto them, the other
ranks' neurons are external populations reading the owners' spike words
directly (the in-process form of the per-step exchange), and every rank's
neuron update finishes before any rank reads another's words.  The rasters
and final membrane potentials of 2- and 3-way splits must equal the unsplit
network's, with input current every step, and with dopamine learning and
rewards (remote pre traces, eligibility of synapses from external neurons).
"""
import numpy as np
import pytest

import simuse_b200 as sg
from simuse_b200 import shard as SH

pytestmark = pytest.mark.gpu

LIF = 1
LEARN = dict(dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=200.0, a_ltp=0.1, a_ltd=0.12, lr=0.5, w_min=-30.0,
             w_max=50.0)


def lif_spec(seed=4, sizes=(1500, 700), k=40):
    rng = np.random.default_rng(seed)
    N = sum(sizes)
    pre = np.repeat(np.arange(N, dtype=np.uint32), k)
    post = rng.integers(0, N, pre.size).astype(np.uint32)
    w = rng.uniform(-20.0, 40.0, pre.size).astype(np.float32)
    d = rng.integers(1, 9, pre.size).astype(np.uint8)
    pops = [SH.PopSpec(LIF, sizes[0], dict(enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 2.0])),
                       {0: rng.uniform(-70.0, -55.0, sizes[0]).astype(np.float32)}),
            SH.PopSpec(LIF, sizes[1], dict(enumerate([0.5, 0.2, -65.0, -52.0, -68.0, 1.0])),
                       {0: rng.uniform(-65.0, -53.0, sizes[1]).astype(np.float32)})]
    return SH.NetSpec(pops, pre, post, w, d)


def run(spec, world, steps, currents, learn):
    shards = [SH.Shard(sg.Network(0), spec, r, world) for r in range(world)]
    for s in shards:
        s.net.build()
        if learn:
            s.net.enable_learning(**LEARN)
    if world > 1:
        SH.link_in_process(shards)
    raster = np.zeros((steps, spec.total), np.int32)
    for t in range(steps):
        for s in shards:
            s.inject(currents[t])
        if world > 1:
            SH.step_in_process(shards)
        else:
            shards[0].net.step(1)
        for s in shards:
            s.spikes(raster[t])
        if learn and t % 50 == 49:
            for s in shards:     # every synapse lives on exactly one rank
                s.net.reward(1.0 if (t // 50) % 2 else -0.6)
    v = np.zeros(spec.total, np.float32)
    for s in shards:
        s.state(0, v)
        s.net.close()
    return raster, v


@pytest.mark.parametrize("learn", [False, True])
def test_split_network_matches_the_unsplit_network(learn):
    sp = lif_spec()
    steps = 300
    cur = np.random.default_rng(9).uniform(0.0, 60.0, (steps, sp.total)).astype(np.float32)
    r1, v1 = run(sp, 1, steps, cur, learn)
    assert r1.sum() > 2000
    for world in (2, 3):
        rw, vw = run(sp, world, steps, cur, learn)
        assert np.array_equal(rw, r1), (world, int(np.nonzero((rw != r1).any(1))[0][0]))
        assert np.array_equal(vw.view(np.uint32), v1.view(np.uint32))


def test_external_population_rules():
    net = sg.Network(0)
    p = net.add_population(LIF, 8)
    x = net.add_external_population(8)
    with pytest.raises(sg.SimuseError):            # no synapses onto external neurons
        net.connect(p, np.array([0], np.uint32), x, np.array([1], np.uint32), np.ones(1, np.float32),
                    np.ones(1, np.uint8))
    net.connect(x, np.array([0], np.uint32), p, np.array([1], np.uint32), np.ones(1, np.float32), np.ones(1, np.uint8))
    net.build()
    with pytest.raises(sg.SimuseError):            # whole steps need the exchange
        net.step(1)
    with pytest.raises(sg.SimuseError):            # no source yet
        net.step_begin()
        net.step_end()
    net.close()
