"""Batches of independent networks stepping as one device network, the
device fixed-out-degree generator, and device-generated input noise.

A batch is one `Network` whose populations are the instances (each with its
own synapses, none between instances): one launch per neuron model and one
scatter launch per step advance all of them.  Ring cells of different
instances are disjoint, so every instance keeps the reference's summation
order and gives the same bits alone or in any batch.
"""
import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

IZH = 2


def _pop_raster(raster, offsets, p, n):
    return raster[:, offsets[p]:offsets[p] + n]


def test_fixed_outdegree_generator_matches_numpy_twin():
    n, k, seed = 1500, 100, 21
    net = sg.Network(0)
    pop = W.add_izhikevich_instance(net, n, seed, device_edges=True, device_noise=False)
    net.build()
    rp, col, w, d = net.graph()
    pre, post, ww = W.fixed_outdegree_edges(n, k, seed, n * 4 // 5, 0.5, -1.0)
    # the device stores each row sorted by post (stable); compare as sorted rows
    order = np.lexsort((post, pre))
    assert np.array_equal(np.diff(rp), np.full(n, k))
    assert np.array_equal(col, post[order])
    assert np.array_equal(w, ww[order])
    assert np.all(d == 1)
    rows = col.reshape(n, k)
    assert all(np.unique(r).size == k for r in rows)          # distinct targets
    assert not np.any(rows == np.arange(n)[:, None])           # no self-loops
    net.close()


def test_device_noise_matches_host_injected_oracle():
    """The device thalamic input equals the host FP64 Box-Muller values fed
    through inject_current, so rasters and states match the oracle."""
    n, seed, steps = 1000, 5, 300
    net = sg.Network(0)
    pop = W.add_izhikevich_instance(net, n, seed, device_edges=True, device_noise=True)
    net.build()
    net.enable_raster(steps)
    net.step(steps)
    gpu = net.read_raster()
    ref = O.Network()
    rp = ref.add_population(IZH, n)
    a, b, c, d = W.izhikevich_params(n, n * 4 // 5, seed)
    for col, v in enumerate([1.0, None, None, None, None, 0.0, 30.0]):
        if v is not None:
            ref.fill_param(rp, col, v)
    for col, v in ((1, a), (2, b), (3, c), (4, d)):
        ref.set_param(rp, col, v)
    ref.fill_state(rp, 0, -65.0)
    ref.set_state(rp, 1, (b * np.float32(-65.0)).astype(np.float32))
    pre, post, w = W.fixed_outdegree_edges(n, min(100, n - 1), seed, n * 4 // 5, 0.5, -1.0)
    ref.connect(rp, pre, rp, post, w, np.ones(pre.size, np.uint8))
    ref.build()
    idx = np.arange(n, dtype=np.uint32)
    cpu = np.zeros((steps, n), np.uint8)
    for t in range(steps):
        ref.inject_current(rp, idx, W.thalamic_input(n, seed, t))
        ref.step(1)
        cpu[t] = ref.spikes(rp)
    assert gpu.sum() > 100
    assert np.array_equal(gpu, cpu)
    assert np.array_equal(net.state(pop, 0), ref.state(rp, 0))
    assert np.array_equal(net.state(pop, 1), ref.state(rp, 1))
    net.close()


def test_batch_equals_instances_alone():
    """Five uneven Izhikevich instances and a LIF population in one batch
    (two neuron models in one work table) give each instance's own bits."""
    sizes, seeds, steps = [500, 1000, 3000, 777, 2048], [1, 2, 3, 4, 5], 250
    batch = sg.Network(0)
    pops = [W.add_izhikevich_instance(batch, n, s) for n, s in zip(sizes, seeds)]
    lif = batch.add_population(sg.LIF, 3000)
    for col, v in enumerate([0.1, 0.05, 25.0, 20.0, 10.0, 2.0]):  # rest above threshold: it fires
        batch.fill_param(lif, col, v)
    batch.set_noise(lif, 99, 40.0)
    batch.build()
    batch.enable_raster(steps)
    batch.step(steps)
    r_batch = batch.read_raster()
    offs = np.concatenate([[0], np.cumsum(sizes + [3000])])
    for p, n, s in zip(pops, sizes, seeds):
        alone = sg.Network(0)
        q = W.add_izhikevich_instance(alone, n, s)
        alone.build()
        alone.enable_raster(steps)
        alone.step(steps)
        r = alone.read_raster()
        assert r.sum() > 10
        assert np.array_equal(r, _pop_raster(r_batch, offs, p, n)), (n, s)
        assert np.array_equal(alone.state(q, 0), batch.state(p, 0))
        alone.close()
    assert r_batch[:, offs[5]:].sum() > 0   # the LIF population is driven by its noise
    batch.close()


def test_noise_settings_validated():
    net = sg.Network(0)
    p = net.add_population(IZH, 10)
    with pytest.raises(sg.SimuseError):
        net.set_noise(p, 1, float("nan"))
    with pytest.raises(sg.SimuseError):
        net.connect_fixed_outdegree(p, p, 10, 1, True, 8, 0.5, -1.0)   # only 9 candidates
    net.close()


def test_noise_change_after_steps_takes_effect():
    """Changing the noise after the step graph was captured is honoured."""
    n = 1000
    a = sg.Network(0)
    pa = W.add_izhikevich_instance(a, n, 3, device_noise=False)
    a.build()
    a.step(64)                      # captures the 32-step graph without noise
    a.set_noise(pa, 3, 5.0, 2.0, split=n * 4 // 5)
    a.step(64)
    b = sg.Network(0)
    pb = W.add_izhikevich_instance(b, n, 3, device_noise=False)
    b.build()
    b.step(64)
    for t in range(64, 128):        # the same input fed from the host
        b.inject_current(pb, np.arange(n, dtype=np.uint32), W.thalamic_input(n, 3, t))
        b.step(1)
    assert np.array_equal(a.state(pa, 0), b.state(pb, 0))
    a.close()
    b.close()


def test_lognormal_outdegree_generator_matches_numpy_twin():
    n, seed = 1200, 8
    net = sg.Network(0)
    p = net.add_population(IZH, n)
    net.connect_lognormal_outdegree(p, p, 100.0, 60.0, seed, True, 960, 0.5, -1.0)
    net.build()
    rp, col, w, d = net.graph()
    pre, post, ww = W.lognormal_outdegree_edges(n, 100.0, 60.0, seed, 960, 0.5, -1.0)
    order = np.lexsort((post, pre))
    assert np.array_equal(col, post[order])
    assert np.array_equal(w, ww[order])
    deg = np.diff(rp)
    assert abs(deg.mean() - 100.0) < 6.0 and abs(deg.std() - 60.0) < 8.0
    for i in range(0, n, 97):                      # distinct targets, no self-loop
        r = col[rp[i]:rp[i + 1]]
        assert np.unique(r).size == r.size and not np.any(r == i)
    net.close()


def _reference_cvs(raster, dt_s):
    """P/kernels/stats/isi.rs:30-66 in float32 (two-pass, sample variance)."""
    n_steps, n = raster.shape
    out = np.zeros(n, np.float32)
    for i in range(n):
        t = np.nonzero(raster[:, i])[0]
        isi = (np.diff(t).astype(np.float32) * np.float32(dt_s) * np.float32(1000.0)).astype(np.float32)
        isi = isi[isi > 0]
        if isi.size >= 2:
            m = np.float32(isi.sum(dtype=np.float32) / np.float32(isi.size))
            var = np.float32(((isi - m) ** 2).sum(dtype=np.float32) / np.float32(isi.size - 1))
            out[i] = np.sqrt(var) / m
    return out


def test_device_rates_and_isi_cv_match_the_raster():
    n, steps = 1000, 600
    net = sg.Network(0)
    p = W.add_izhikevich_instance(net, n, 17)
    net.build()
    net.step(20)
    net.enable_neuron_stats()
    net.enable_raster(steps)
    net.step(steps)
    raster = net.read_raster()
    rates, cv, mean_ms, nst = net.neuron_stats(p, 1.0)
    assert nst == steps
    counts = raster.sum(axis=0)
    assert np.array_equal(np.rint(rates * steps * 1e-3).astype(int), counts)
    ref = _reference_cvs(raster, 1e-3)
    has = ref > 0
    assert has.sum() > 100
    assert np.allclose(cv[has], ref[has], rtol=1e-4)
    assert np.all(cv[~has] == 0)
    net.close()


def test_outdegree_generator_delays_types_and_stdp_flags():
    n, k, seed = 800, 40, 5
    net = sg.Network(0)
    p = net.add_population(sg.HH, n)
    ke = net.register_expone(5.0, 0.0, 0.01)
    ki = net.register_expone(5.0, -80.0, 0.01)
    net.stdp_config(0.01, 20.0, 20.0, 0.01, 0.0105, 0.0, 1.0)
    net.connect_fixed_outdegree(p, p, k, seed, True, 640, 0.5, 0.5, True, 3, d_max=17,
                                syn_type_exc=ke, syn_type_inh=ki, stdp_exc=True)
    net.build()
    rp, col, w, d = net.graph()
    pre, post, _ = W.fixed_outdegree_edges(n, k, seed, 640, 0.5, 0.5)
    dd = W.fixed_outdegree_delays(n, k, seed, 3, 17)
    order = np.lexsort((post, pre))
    assert np.array_equal(d, dd[order])
    assert d.min() >= 3 and d.max() <= 17 and np.unique(d).size == 15
    net.close()


def test_hh_stdp_workload_builds_and_runs():
    net = sg.Network(0)
    W.add_hh_stdp(net, n=5000)
    net.build()
    net.step(500)
    assert net.events_total > 0
    assert net.stdp_drift != 0.0
    net.close()
