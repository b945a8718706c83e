"""Parity at the benchmark's full sizes.

The headline network (1,000,000 LIF neurons, fixed in-degree 1000: 1e9
synapses, delays 1-20 steps, one Poisson source per neuron) is built on the
device and on the oracle from the same seeded generator and stepped from its
initial state; spike rasters, membrane and refractory bits and the event
count must be identical.  This exercises what small networks do not: every
scatter block and warp busy, 21 ring slots, rows of ~1000 synapses, the
deferred drive on a million neurons.  Both variants of the configuration run:
the driven one (4000 Hz x 100, ~3.8e6 events per step) and the literal one
(2000 Hz x 20, silent apart from the Poisson events).

The HH + pair-STDP network at its stated size (100,000 neurons, lognormal
out-degree (200, 80), ~2e7 synapses) runs 2,000 steps (20 ms) on both: the
test reports the first step whose raster differs, if any, and requires none,
with membrane bits and STDP-updated weights equal at the end.
"""
import os

import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _oracle_lif(spec):
    O.set_threads(os.cpu_count() or 1)
    c = O.Network(0)
    p = c.add_population(O.LIF, spec["n"])
    for col, v in enumerate(W.LIF_PARAMS):
        c.fill_param(p, col, v)
    c.set_state(p, 0, spec["v0"])
    first = c.add_poisson_sources(spec["n"], spec["ext_rate_hz"], spec["dt"], seed0=0)
    c.connect_poisson_one_to_one(first, spec["n"], p, spec["ext_weight"], 1)
    c.build_fixed_indegree(p, p, spec["k_in"], spec["seed"], spec["n_exc"], spec["w_exc"], spec["w_inh"],
                           spec["d_min"], spec["d_max"])
    return c, p


@pytest.mark.parametrize("variant,steps", [("driven", 250), ("literal", 400)])
def test_lif_1m_prefix_bit_identical(variant, steps):
    kw = (dict(ext_rate_hz=4000.0, ext_weight=100.0) if variant == "driven"
          else dict(ext_rate_hz=2000.0, ext_weight=20.0))
    spec = W.lif_balanced(n=1_000_000, k_in=1000, seed=1, **kw)
    g = sg.Network(0)
    gp = W.build_lif(g, spec)
    g.build()
    assert g.num_synapses == 10**9
    c, cp = _oracle_lif(spec)
    chunk = 50
    spikes = 0
    for k in range(0, steps, chunk):
        g.enable_raster(chunk)
        g.step(chunk)
        rg = g.read_raster()
        rc = c.step(chunk, record=True)
        spikes += int(rg.sum())
        if not np.array_equal(rg, rc):
            bad = np.nonzero((rg != rc).any(axis=1))[0]
            pytest.fail(f"raster differs first at step {k + int(bad[0])}")
    print(f"LIF 1M {variant}: {steps} steps, {spikes} spikes, {g.events_total} events, identical")
    if variant == "driven":
        assert spikes > 1000 * steps  # the recurrent network is active
    for col in (0, 1):
        assert np.array_equal(g.state(gp, col).view(np.uint32), c.state(cp, col).view(np.uint32)), col
    assert g.events_total == c.events
    g.close()


def test_hh_stdp_100k_prefix_bit_identical():
    n, steps = 100_000, 2000
    g = sg.Network(0)
    gp = W.add_hh_stdp(g, n, w_max=0.01)
    g.build()
    rp, col, w, d = g.graph()
    st, pl = g.graph_types()
    assert g.num_synapses > 15_000_000
    O.set_threads(os.cpu_count() or 1)
    c = O.Network(0)
    cp = W.add_hh_stdp(c, n, w_max=0.01, edges=(rp, col, w, d, st, pl))
    c.build()
    first, spikes = None, 0
    for k in range(0, steps, 500):
        g.enable_raster(500)
        g.step(500)
        rg = g.read_raster()
        rc = c.step(500, record=True)
        spikes += int(rg.sum())
        bad = np.nonzero((rg != rc).any(axis=1))[0]
        if bad.size and first is None:
            first = k + int(bad[0])
    print(f"HH+STDP 100k: {steps} steps, {spikes} spikes; first divergent step: {first}")
    assert spikes > 0
    assert first is None
    assert np.array_equal(g.state(gp, 0).view(np.uint32), c.state(cp, 0).view(np.uint32))
    assert np.array_equal(g.weights().view(np.uint32), c.weights().view(np.uint32))
    g.close()
