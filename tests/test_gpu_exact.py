"""The exact-sum scatter path.

When every weight that reaches a ring is a multiple of one power of two and
no post's weights can sum past 24 bits of mantissa at that scale, every
partial sum of a ring cell is exact in FP32: float addition on the rings is
associative and the order of the adds cannot change a bit.  The network then
takes the pre-centric scatter (each spiking row read once, every event added
to its ring cell in L2 with red.global.add, in any order); everything else
keeps the reference's order.  These tests check which networks take the path
and that it gives the oracle's bits, on a network where every neuron fires
every step and when the rings are read back between steps.
"""
import numpy as np
import pytest

import oracle as O
import scenarios as S
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

LIF = 1


def _balanced(net, w_exc=20.0, g=5.0, ext_w=100.0, n=2000):
    spec = W.lif_balanced(n=n, k_in=100, seed=3, ext_rate_hz=4000.0, ext_weight=ext_w, w_exc=w_exc, g=g)
    return W.build_lif(net, spec, device_generator=isinstance(net, sg.Network))


def _mode(**kw):
    net = sg.Network(0)
    _balanced(net, **kw)
    net.build()
    m = net.scatter_mode
    net.close()
    return m


def test_path_selection():
    assert _mode() == "exact"                               # 20, -100, Poisson 100
    assert _mode(w_exc=2.5, g=4.0, ext_w=0.125) == "exact"  # multiples of 2^-3
    assert _mode(w_exc=0.1) == "ordered"                    # 0.1 is not a dyadic fraction of small size
    assert _mode(w_exc=2.0 ** 20) == "ordered"              # integer, but 100 inputs pass 2^23
    net = sg.Network(0)
    _balanced(net)
    net.set_deterministic(False)
    net.build()
    assert net.scatter_mode == "atomic"
    net.close()


def test_stdp_keeps_the_ordered_path():
    net = sg.Network(0)
    p = net.add_population(LIF, 64)
    net.stdp_config(0.1, 20.0, 20.0, 0.01, 0.0105, 0.0, 4.0)
    pre = np.arange(64, dtype=np.uint32)
    net.connect(p, pre, p, (pre + 1) % 64, np.full(64, 2.0, np.float32), np.ones(64, np.uint8), stdp=True)
    net.build()
    assert net.scatter_mode == "ordered"
    net.close()


def _dense(net, n=4096, k=512, steps=30):
    """Every neuron fires every step (dt * inv_tau = 1 puts v at rest + input,
    rest above threshold, no refractory time): 2M events a step over two
    delays, many of them onto the same ring cells within a step."""
    p = net.add_population(LIF, n)
    for col, v in enumerate([1.0, 1.0, 25.0, 20.0, 10.0, 0.0]):
        net.fill_param(p, col, v)
    net.fill_state(p, 0, 30.0)
    rng = np.random.default_rng(7)
    post = np.repeat(np.arange(n, dtype=np.uint32), k)
    pre = rng.integers(0, n, post.size).astype(np.uint32)
    w = rng.choice(np.array([1.0, 2.0, -1.0, 3.0], np.float32), post.size)
    d = rng.integers(1, 3, post.size).astype(np.uint8)
    order = np.lexsort((post, pre))
    net.connect(p, pre[order], p, post[order], w[order], d[order])
    net.build()
    raster = []
    for _ in range(steps):
        net.step(1)
        raster.append(net.spikes(p).copy())
    return net, p, np.array(raster)


def test_exact_dense_firing_matches_the_oracle():
    g, gp, rg = _dense(sg.Network(0))
    assert g.scatter_mode == "exact"
    c, cp, rc = _dense(O.Network(0))
    assert rg.sum() > rg.size // 2
    assert np.array_equal(rg, rc)
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert np.array_equal(g.ring(0).view(np.uint32), c.ring(0).view(np.uint32))
    g.close()


def test_exact_ring_readback_between_steps():
    """Reading the rings between steps (which first adds the deferred drive
    of the last step to them) and stepping on from there gives the same bits
    as never having read them."""
    g = sg.Network(0)
    gp = _balanced(g)
    g.build()
    c = O.Network(0)
    cp = _balanced(c)
    c.build()
    assert g.scatter_mode == "exact"
    for chunk in (37, 1, 90):
        g.enable_raster(chunk)
        g.step(chunk)
        rg = g.read_raster()
        rc = c.step(chunk, record=True)
        assert np.array_equal(rg, rc)
        assert np.array_equal(g.ring(0).view(np.uint32), c.ring(0).view(np.uint32))
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    g.close()


def test_autotuned_schedule_keeps_the_oracle_bits():
    """sg_autotune runs the network's next steps under every candidate
    schedule of the pre-centric scatter (four stage-ring shapes and the warp
    walk) and keeps the fastest; the steps are ordinary simulation steps and
    every schedule gives the same bits."""
    g = sg.Network(0)
    gp = _balanced(g)
    g.build()
    c = O.Network(0)
    cp = _balanced(c)
    c.build()
    rep = g.autotune(steps=20)
    assert rep["fixed_ms_per_step"] > 0 and rep["tuned_ms_per_step"] > 0
    assert rep["tuned_ms_per_step"] <= rep["fixed_ms_per_step"]
    done = g.step_counter            # 27 candidates (9 schedules x 1-3 blocks per SM) x (20 warm-up + 20 timed)
    assert done == 27 * 40
    c.step(done)
    g.enable_raster(50)
    g.step(50)
    rg = g.read_raster()
    rc = c.step(50, record=True)
    assert np.array_equal(rg, rc)
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert g.events_total == c.events
    g.close()
