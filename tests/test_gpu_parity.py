"""Parity of the CUDA step (through the C ABI) with the CPU oracle and the
reference's pins.  Bit-exact for spikes, rings and FP32 state wherever the
reference arithmetic is deterministic (LIF, Izhikevich, HH-RK4 with the
shared exp, kinetics, pair STDP weights); stated tolerances elsewhere."""
import numpy as np
import pytest

import oracle as O
import scenarios as S

pytestmark = pytest.mark.gpu


def gpu():
    from simuse_b200 import Network
    return Network(0)


def cpu():
    return O.Network(0)


PINS = S.PINS


@pytest.mark.parametrize("cfg", PINS["lif_spike_counts"]["configs"], ids=lambda c: c["label"])
def test_lif_golden_spike_counts_gpu(cfg):
    pin = PINS["lif_spike_counts"]
    counts = S.lif_pin_counts(gpu, cfg, n=pin["n"], t_ms=pin["t_ms"], on_ms=pin["on_ms"])
    assert np.all(counts == int(cfg["ref_spikes"]))


@pytest.mark.parametrize("cfg", PINS["izh_patterns"]["configs"], ids=lambda c: c["label"])
def test_izhikevich_patterns_gpu_equal_oracle(cfg):
    per_g, cv_g = S.izh_pattern(gpu, cfg, PINS["izh_patterns"])
    per_c, cv_c = S.izh_pattern(cpu, cfg, PINS["izh_patterns"])
    assert np.array_equal(per_g, per_c)
    assert cv_g == cv_c
    assert cfg["min_spikes"] <= per_g.mean() <= cfg["max_spikes"]


@pytest.mark.parametrize("n", PINS["delay_arrival"]["sizes"])
def test_delay_arrival_gpu(n):
    delays = PINS["delay_arrival"]["delays"]
    d = [delays[i % len(delays)] for i in range(n)]
    a0, raster = S.delay_arrival(gpu, n, d)
    assert np.all(a0 == 1)
    for i, dl in enumerate(d):
        expect = np.zeros(raster.shape[0], np.int32)
        expect[max(dl, 1)] = 1
        assert np.array_equal(raster[:, i], expect), (i, dl)


@pytest.mark.parametrize("case", PINS["push"]["cases"], ids=lambda c: c["name"])
def test_push_slot_arithmetic_gpu(case):
    ring, spikes = S.push_case(gpu, case)
    expect = np.zeros_like(ring)
    for slot, post, val in case["expect"]:
        expect[slot, post] += val
    assert np.array_equal(ring, expect)


@pytest.mark.parametrize("seed", [7, 8, 9])
def test_collision_order_bit_exact(seed):
    # random non-integer weights converging on shared cells: the ring must
    # hold the reference's sequential sums bit for bit
    rg, ring_g, vg = S.random_collision_net(gpu, seed=seed)
    rc, ring_c, vc = S.random_collision_net(cpu, seed=seed)
    assert rg.sum() > 0
    assert np.array_equal(rg, rc)
    assert np.array_equal(ring_g.view(np.uint32), ring_c.view(np.uint32))
    assert np.array_equal(vg.view(np.uint32), vc.view(np.uint32))


def test_izhikevich_pulse_network_bit_identical():
    # the plain Izhikevich pulse-coupled network, full 1000 steps
    import simuse_b200.workloads as W
    spec = W.izhikevich_pulse()
    rasters = []
    finals = []
    for mk in (gpu, cpu):
        net = mk()
        pop = W.build_izhikevich(net, spec)
        idx = np.arange(spec["n"], dtype=np.uint32)
        r = []
        for t in range(spec["steps"]):
            net.inject_current(pop, idx, W.izhikevich_input(spec, t))
            net.step(1)
            r.append(net.spikes(pop).copy())
        rasters.append(np.array(r))
        finals.append((net.state(pop, 0), net.state(pop, 1)))
    assert rasters[0].sum() > 1000
    assert np.array_equal(rasters[0], rasters[1])
    for a, b in zip(finals[0], finals[1]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_izhikevich_raster_recording_and_graph_replay():
    # many steps per call (CUDA-graph replay) with on-device raster
    import simuse_b200.workloads as W
    spec = W.izhikevich_pulse(noise=False)
    g = gpu()
    pop = W.build_izhikevich(g, spec)
    g.fill_state(pop, 0, -50.0)
    g.enable_raster(200)
    g.step(200)
    rg = g.read_raster()
    c = cpu()
    popc = W.build_izhikevich(c, spec)
    c.fill_state(popc, 0, -50.0)
    rc = c.step(200, record=True)
    assert rg.shape == rc.shape
    assert np.array_equal(rg, rc)
    assert g.step_counter == 200


def test_lif_balanced_small_bit_identical():
    gnet, gpop, rg = S.lif_small_balanced(gpu, device_generator=True)
    cnet, cpop, rc = S.lif_small_balanced(cpu, device_generator=False)
    # the device generator builds exactly the numpy-restated CSR
    for a, b in zip(gnet.graph(), cnet.graph()):
        assert np.array_equal(a, b)
    assert rg.sum() > 100
    assert np.array_equal(rg, rc)
    assert np.array_equal(gnet.state(gpop, 0).view(np.uint32), cnet.state(cpop, 0).view(np.uint32))
    assert gnet.events_total == cnet.events


def test_atomic_mode_matches_when_sums_are_exact():
    # integer-valued weights: every order gives the same sums, so the
    # non-deterministic atomic scatter must agree exactly as well
    from simuse_b200 import workloads as W
    spec = W.lif_balanced(n=2000, k_in=100, seed=3, ext_rate_hz=4000.0, ext_weight=100.0)
    outs = []
    for det in (True, False):
        net = gpu()
        pop = W.build_lif(net, spec)
        net.set_deterministic(det)
        net.build()
        net.enable_raster(300)
        net.step(300)
        outs.append(net.read_raster())
    assert np.array_equal(outs[0], outs[1])


def test_inject_duplicates_apply_in_order():
    vals = np.array([1e8, 1.0, -1e8, 0.5], np.float32)
    idx = np.array([3, 3, 3, 3], np.uint32)
    rings = []
    for mk in (gpu, cpu):
        net = mk()
        p = net.add_population(S.LIF, 5)
        net.fill_param(p, 0, 0.1)
        net.build()
        net.inject_current(p, idx, vals)
        rings.append(net.ring(0))
    assert np.array_equal(rings[0], rings[1])


def test_contract_violations_gpu():
    from simuse_b200 import SimuseError
    net = gpu()
    p = net.add_population(S.LIF, 4)
    with pytest.raises(SimuseError):
        net.connect(p, [0], p, [9], [1.0], [0])
    with pytest.raises(SimuseError):
        net.connect(p, [0], p, [1], [1.0], [32])
    with pytest.raises(SimuseError):
        net.connect(p, [0], p, [1], [float("inf")], [0])
    with pytest.raises(SimuseError):
        net.step(1)
    net.build()
    with pytest.raises(SimuseError) as e:
        net.build()
    assert e.value.code == -2
    with pytest.raises(SimuseError):
        net.inject_current(p, [4], [1.0])
    with pytest.raises(SimuseError):
        net.fill_param(p, 6, 0.0)


def test_empty_network_gpu():
    net = gpu()
    net.build()
    net.step(5)
    assert net.step_counter == 5


def test_multiple_populations_and_padding():
    # populations of sizes that are not multiples of 32 (padded device layout)
    rng = np.random.default_rng(1)
    outs = []
    for mk in (gpu, cpu):
        net = mk()
        pops = [net.add_population(S.LIF, n) for n in (5, 33, 70)]
        for p in pops:
            for col, v in enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 1.0]):
                net.fill_param(p, col, v)
            net.fill_state(p, 0, -60.0)
        r = np.random.default_rng(2)
        for a in pops:
            for b in pops:
                na, nb = net._sizes[a], net._sizes[b]
                k = 3 * na
                net.connect(a, r.integers(0, na, k), b, r.integers(0, nb, k),
                            r.uniform(5, 40, k).astype(np.float32), r.integers(0, 6, k))
        net.build()
        res = []
        for t in range(150):
            for p in pops:
                n = net._sizes[p]
                net.inject_current(p, np.arange(n, dtype=np.uint32),
                                   np.full(n, 18.0 + (t % 7), np.float32))
            net.step(1)
            res.append(np.concatenate([net.spikes(p) for p in pops]))
        outs.append((np.array(res), net.ring(0)))
    assert outs[0][0].sum() > 50
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
