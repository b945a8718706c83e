"""Deferred drive: a population driven one-to-one by Poisson sources (source
seed0 + i onto neuron i, one rate and weight, delay <= 1) takes that drive in
the neuron kernel of the next step instead of the scatter.  A delay-1 event
of step t is the last add into slot t + 1 before that slot is read, so adding
it to the value read gives the ring's float sums; an inject_current or a ring
readback in between first folds it into the ring, where the reference keeps
it (P/api/net/network/step.rs:166-185, build.rs:243-275).

These tests compare rasters, membrane bits, event counts and ring contents
with the oracle while inputs are injected and rings read between steps, on
the exact-sum (pre-centric) and the ordered scatter paths, and on networks
mixing deferred and scattered drive.
"""
import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

LIF = 1


def _balanced(net, w_exc, ext_w, n=3000):
    spec = W.lif_balanced(n=n, k_in=100, seed=5, ext_rate_hz=4000.0, ext_weight=ext_w, w_exc=w_exc, g=5.0)
    return W.build_lif(net, spec, device_generator=isinstance(net, sg.Network))


def _run_pair(g, gp, c, cp, script, n):
    """Runs `script` (a list of ("step", k) / ("inject", seed) / ("ring",))
    on the device network g and the oracle c, comparing as it goes."""
    for item in script:
        if item[0] == "step":
            k = item[1]
            g.enable_raster(k)
            g.step(k)
            rg = g.read_raster()
            rc = c.step(k, record=True)
            assert np.array_equal(rg, rc), f"raster differs in {item}"
        elif item[0] == "inject":
            rng = np.random.default_rng(item[1])
            idx = np.sort(rng.choice(n, size=n // 3, replace=False)).astype(np.uint32)
            vals = (rng.standard_normal(idx.size) * 7.3).astype(np.float32)
            g.inject_current(gp, idx, vals)
            c.inject_current(cp, idx, vals)
        else:
            assert np.array_equal(g.ring(0).view(np.uint32), c.ring(0).view(np.uint32)), "ring differs"
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert g.events_total == c.events


SCRIPT = [("step", 40), ("inject", 1), ("step", 1), ("ring",), ("step", 33), ("inject", 2), ("ring",),
          ("inject", 3), ("step", 2), ("step", 64), ("ring",), ("inject", 4), ("step", 20)]


@pytest.mark.parametrize("w_exc,ext_w,mode", [(20.0, 100.0, "exact"), (0.1, 100.3, "ordered")])
def test_deferred_drive_with_inject_and_readback(w_exc, ext_w, mode):
    n = 3000
    g = sg.Network(0)
    gp = _balanced(g, w_exc, ext_w, n)
    g.build()
    assert g.scatter_mode == mode
    c = O.Network(0)
    cp = _balanced(c, w_exc, ext_w, n)
    c.build()
    _run_pair(g, gp, c, cp, SCRIPT, n)
    g.close()


def _mixed(net, n=2048, w_exc=20.0):
    """Population A: one-to-one drive (deferred).  Population B: drive on
    every other neuron only, plus a delay-3 source onto a few neurons (both
    stay in the scatter).  Recurrent synapses among and between them."""
    a = net.add_population(LIF, n)
    b = net.add_population(LIF, n)
    for p in (a, b):
        for col, v in enumerate(W.LIF_PARAMS):
            net.fill_param(p, col, v)
        net.set_state(p, 0, (10.0 + 10.0 * W.uniform01(9, p, np.arange(n, dtype=np.uint64))).astype(np.float32))
    first = net.add_poisson_sources(n, 4000.0, 0.1, seed0=100)
    net.connect_poisson_one_to_one(first, n, a, 100.0, 1)
    half = np.arange(0, n, 2, dtype=np.uint32)
    fb = net.add_poisson_sources(half.size, 4000.0, 0.1, seed0=50_000)
    net.connect_poisson_one_to_one(fb, half.size, b, 100.0, 1, posts=half)
    s3 = net.add_poisson_source(3000.0, 0.1, 7)
    few = np.arange(0, n, 97, dtype=np.uint32)
    net.connect_poisson_source(s3, b, few, np.full(few.size, 60.0, np.float32), np.full(few.size, 3, np.uint8))
    rng = np.random.default_rng(3)
    m = n * 60
    for src, dst in ((a, a), (a, b), (b, a)):
        pre = rng.integers(0, n, m).astype(np.uint32)
        post = rng.integers(0, n, m).astype(np.uint32)
        w = np.where(pre < n * 4 // 5, w_exc, -100.0).astype(np.float32)
        d = rng.integers(1, 8, m).astype(np.uint8)
        net.connect(src, pre, dst, post, w, d)
    return a, b


@pytest.mark.parametrize("w_exc,mode", [(20.0, "exact"), (20.1, "ordered")])
def test_mixed_deferred_and_scattered_drive(w_exc, mode):
    n = 2048
    g = sg.Network(0)
    ga, gb = _mixed(g, n, w_exc)
    g.build()
    assert g.scatter_mode == mode
    c = O.Network(0)
    ca, cb = _mixed(c, n, w_exc)
    c.build()
    for k in (1, 30, 45, 2):
        g.enable_raster(k)
        g.step(k)
        rg = g.read_raster()
        rc = c.step(k, record=True)
        assert np.array_equal(rg, rc)
        assert np.array_equal(g.ring(0).view(np.uint32), c.ring(0).view(np.uint32))
    for gp, cp in ((ga, ca), (gb, cb)):
        assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert g.events_total == c.events
    g.close()


def test_ring_clear_drops_the_deferred_drive():
    """After sg_ring_clear nothing is pending: the next step reads an empty
    slot (no deferred event of the previous step), as a freshly built network
    with the same state does on its first step."""
    n = 1024

    def make(net):
        p = net.add_population(LIF, n)
        for col, v in enumerate(W.LIF_PARAMS):
            net.fill_param(p, col, v)
        net.fill_state(p, 0, 0.0)
        first = net.add_poisson_sources(n, 9000.0, 0.1, seed0=0)  # p = 0.9: most sources fire each step
        net.connect_poisson_one_to_one(first, n, p, 1.0, 1)
        return p

    g = sg.Network(0)
    p = make(g)
    g.build()
    g.step(5)
    g.clear_rings()
    assert not g.ring(0).any()
    v0 = g.state(p, 0).copy()
    g.step(1)
    c = O.Network(0)
    cp = make(c)
    c.build()
    c.set_state(cp, 0, v0)
    c.step(1)
    assert np.array_equal(g.state(p, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert not np.array_equal(v0, g.state(p, 0))  # the step did integrate
    g.close()
