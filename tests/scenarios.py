"""Scenarios that drive any backend with the reference's builder/step API.

A backend is either the product (simuse_b200.Network, CUDA through the C ABI)
or the oracle (oracle.Network, the CPU restatement); both expose the same
method names, so one scenario function runs on both and the results are
compared bit for bit.
"""
from __future__ import annotations

import json
import os

import numpy as np

PINS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))

LIF, IZH, GPEA, HH = 1, 2, 3, 4


def lif_pin_counts(make_net, cfg, n=8, t_ms=500.0, on_ms=10.0):
    """tests/lif_vs_neuron.rs:35-73: n LIF neurons, current I switched on at
    10 ms (fed through inject_current), spikes counted over t_ms."""
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([cfg["dt"], 1.0 / cfg["tau_m"], cfg["v_rest"], cfg["v_thresh"],
                             cfg["v_reset"], cfg["tau_ref"]]):
        net.fill_param(p, col, v)
    net.fill_state(p, 0, cfg["v_rest"])
    net.build()
    steps = int(t_ms / cfg["dt"])
    on = int(on_ms / cfg["dt"])
    idx = np.arange(n, dtype=np.uint32)
    cur = np.full(n, cfg["i_syn"], np.float32)
    total = np.zeros(n, np.int64)
    for s in range(steps):
        if s >= on:
            net.inject_current(p, idx, cur)
        net.step(1)
        total += net.spikes(p)
    return total


def izh_pattern(make_net, cfg, pin):
    """tests/izhikevich_vs_neuron.rs:91-150: spike count and ISI CV."""
    n, dt = pin["n"], pin["dt"]
    net = make_net()
    p = net.add_population(IZH, n)
    for col, v in enumerate([dt, cfg["a"], cfg["b"], cfg["c"], cfg["d"], pin["tau_ref"], pin["v_thresh"]]):
        net.fill_param(p, col, v)
    net.fill_state(p, 0, cfg["c"])
    net.build()
    steps = int(pin["t_ms"] / dt)
    on = int(pin["on_ms"] / dt)
    idx = np.arange(n, dtype=np.uint32)
    cur = np.full(n, cfg["i_syn"], np.float32)
    per = np.zeros(n, np.int64)
    times = []
    for s in range(steps):
        if s >= on:
            net.inject_current(p, idx, cur)
        net.step(1)
        sp = net.spikes(p)
        per += sp
        for _ in range(int(sp.sum())):
            times.append(np.float32(s) * np.float32(dt))
    isi = np.diff(np.array(times, np.float32)) if len(times) > 1 else np.array([], np.float32)
    cv = 0.0
    if isi.size > 2:
        mean = isi.mean()
        cv = float(np.sqrt(((isi - mean) ** 2).mean()) / max(mean, 1e-6))
    return per, cv


def delay_arrival(make_net, n, delays):
    """tests/network_delays.rs:71-136: A[i] -> B[i] with delays[i], every A
    neuron forced to spike at step 0; returns B's raster [steps][n]."""
    pin = PINS["delay_arrival"]
    net = make_net()
    a = net.add_population(LIF, n)
    b = net.add_population(LIF, n)
    for pop in (a, b):
        for col, v in enumerate(pin["lif_params"]):
            net.fill_param(pop, col, v)
        net.fill_state(pop, 0, pin["v0"])
    idx = np.arange(n, dtype=np.uint32)
    net.connect(a, idx, b, idx, np.full(n, pin["w_strong"], np.float32), np.asarray(delays, np.uint8))
    net.build()
    net.fill_state(a, 0, pin["force_v"])
    raster = []
    a0 = None
    for s in range(pin["run_steps"]):
        net.step(1)
        if s == 0:
            a0 = net.spikes(a).copy()
        raster.append(net.spikes(b).copy())
    return a0, np.array(raster)


def push_case(make_net, case):
    """A push_spikes unit case (P/api/net/push.rs:300-499) run through the
    whole step: the `active` neurons are forced to spike at step `step`, the
    ring is read right after that step."""
    n = case["n"]
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([0.5, 0.001, -70.0, -54.0, -70.0, 2.0]):
        net.fill_param(p, col, v)
    net.fill_state(p, 0, -70.0)
    net.connect(p, np.array(case["from"], np.uint32), p, np.array(case["to"], np.uint32),
                np.array(case["w"], np.float32), np.array(case["d"], np.uint8))
    net.build()
    if case["step"]:
        net.step(case["step"])
    v = np.full(n, -70.0, np.float32)
    v[np.array(case["active"], dtype=np.int64)] = 100.0
    net.set_state(p, 0, v)
    net.step(1)
    return net.ring(0), net.spikes(p)


def random_collision_net(make_net, n=64, seed=7, steps=12, k=48):
    """Many spiking pres hitting the same posts in the same slots with
    random (non-integer) weights: per-cell summation order matters."""
    rng = np.random.default_rng(seed)
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([0.5, 0.5, -70.0, -54.0, -70.0, 0.0]):
        net.fill_param(p, col, v)
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    post = rng.integers(0, n, n * k).astype(np.uint32)
    w = (rng.standard_normal(n * k) * 7.3).astype(np.float32)
    d = rng.integers(0, 4, n * k).astype(np.uint8)
    net.connect(p, pre, p, post, w, d)
    net.build()
    v0 = rng.uniform(-70, 30, n).astype(np.float32)
    net.set_state(p, 0, v0)
    rasters, rings = [], []
    for s in range(steps):
        net.inject_current(p, np.arange(n, dtype=np.uint32), rng.uniform(0, 60, n).astype(np.float32))
        net.step(1)
        rasters.append(net.spikes(p).copy())
        rings.append(net.ring(0).copy())
    return np.array(rasters), np.array(rings), net.state(p, 0)


def lif_small_balanced(make_net, n=2000, k_in=100, steps=300, device_generator=False, ext_w=100.0,
                       ext_rate=4000.0, seed=3):
    """A downscaled balanced LIF network with Poisson drive."""
    from simuse_b200 import workloads as W
    spec = W.lif_balanced(n=n, k_in=k_in, seed=seed, ext_rate_hz=ext_rate, ext_weight=ext_w)
    net = make_net()
    pop = W.build_lif(net, spec, device_generator=device_generator)
    net.build()
    raster = []
    for s in range(steps):
        net.step(1)
        raster.append(net.spikes(pop).copy())
    return net, pop, np.array(raster)


def hh_network(make_net, n=240, k_out=12, steps=400, seed=11, stdp=True, precision_net=None):
    """A downscaled HH network with conductance synapses and pair STDP: HH
    neurons (squid axon, RK4, dt 0.01 ms), ExpOne E (0 mV) / I (-80 mV)
    synapses tau 5 ms, lognormal out-degree, 80/20 E/I, bias N(10, 2),
    weights U(0, 0.5) nS, STDP on E synapses (tau 20 ms, A+ 0.01, A- 0.0105,
    clip [0, 1])."""
    rng = np.random.default_rng(seed)
    dt = 0.01
    net = make_net()
    n_e = n * 4 // 5
    pe = net.add_population(HH, n_e)
    pi = net.add_population(HH, n - n_e)
    for p, cnt in ((pe, n_e), (pi, n - n_e)):
        for col, v in enumerate([dt, 1.0, 120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 0.0, 0.0]):
            net.fill_param(p, col, v)
        net.set_param(p, 8, rng.normal(10.0, 2.0, cnt).astype(np.float32))
        v0 = rng.uniform(-70, -60, cnt).astype(np.float32)
        net.set_state(p, 0, v0)
        net.fill_state(p, 1, 0.0529)
        net.fill_state(p, 2, 0.5961)
        net.fill_state(p, 3, 0.3177)
    ke = net.register_expone(5.0, 0.0, dt)
    ki = net.register_expone(5.0, -80.0, dt)
    net.stdp_config(dt, 20.0, 20.0, 0.01, 0.0105, 0.0, 1.0)
    sigma = np.sqrt(np.log(1 + (0.4) ** 2))
    for src_pop, cnt, st, plastic in ((pe, n_e, ke, stdp), (pi, n - n_e, ki, False)):
        deg = np.clip(np.round(rng.lognormal(np.log(k_out) - sigma ** 2 / 2, sigma, cnt)), 1, None).astype(int)
        pre = np.repeat(np.arange(cnt), deg).astype(np.uint32)
        tot = pre.size
        tgt = rng.integers(0, n, tot)
        for dst_pop, lo, hi in ((pe, 0, n_e), (pi, n_e, n)):
            sel = (tgt >= lo) & (tgt < hi)
            k = int(sel.sum())
            if k == 0:
                continue
            net.connect(src_pop, pre[sel], dst_pop, (tgt[sel] - lo).astype(np.uint32),
                        rng.uniform(0, 0.5, k).astype(np.float32), rng.integers(1, 30, k).astype(np.uint8),
                        syn_types=np.full(k, st, np.uint8), stdp=plastic)
    net.build()
    rast = []
    for s in range(steps):
        net.step(1)
        rast.append(np.concatenate([net.spikes(pe), net.spikes(pi)]))
    return net, (pe, pi), np.array(rast)


def gpea_network(make_net, n=64, steps=300, seed=5):
    """A small GPEA population with random synapses and a current step."""
    rng = np.random.default_rng(seed)
    net = make_net()
    p = net.add_population(GPEA, n)
    params = [0.025, 24.0, 1.0, 0.0, 2513.2742, 50.0, 10.0, 0.05, -60.0, 0.5, 1.0, 2.0, 3.355e-11, 0.1]
    for col, v in enumerate(params):
        net.fill_param(p, col, v)
    net.set_state(p, 0, rng.uniform(-65, -55, n).astype(np.float32))
    for col, v in ((1, 0.05), (2, 0.6), (3, 0.3), (4, 0.1), (5, 0.5), (6, 5e-5), (7, 0.0), (8, 1.0)):
        net.fill_state(p, col, v)
    k = n * 6
    net.connect(p, rng.integers(0, n, k).astype(np.uint32), p, rng.integers(0, n, k).astype(np.uint32),
                rng.uniform(0, 8, k).astype(np.float32), rng.integers(1, 8, k).astype(np.uint8))
    net.build()
    idx = np.arange(n, dtype=np.uint32)
    rast, v = [], []
    for s in range(steps):
        if s > 20:
            net.inject_current(p, idx, np.full(n, 12.0, np.float32))
        net.step(1)
        rast.append(net.spikes(p).copy())
    return net, p, np.array(rast)


def tm_drive(make_net, steps=500):
    """P/api/net/network/tests.rs:530-575 (plastic_synapse_depresses_repeated_drive):
    three LIF neurons with the test's parameters, a fast-refractory pre
    driven by 100 every step, pre -> post 1 static (weight 100, delay 0) and
    pre -> post 2 through a depressing Tsodyks-Markram synapse (U0 0.5,
    tau_rec 10 ms, dt 0.5).  Returns (spikes of post 1, of post 2)."""
    net = make_net()
    p = net.add_population(LIF, 3)
    for col, v in enumerate([0.5, 0.1, -70.0, -65.0, -70.0, 1.0]):  # v_thresh -65, tau_ref 1
        net.fill_param(p, col, v)
    net.fill_state(p, 0, -70.0)
    plast = net.register_plasticity(0.5, 10.0, 0.5)
    assert plast == 1
    net.connect(p, np.array([0, 0], np.uint32), p, np.array([1, 2], np.uint32), np.array([100.0, 100.0], np.float32),
                np.zeros(2, np.uint8), plast_types=np.array([0, plast], np.uint8))
    net.build()
    fired = np.zeros(3, np.int64)
    for _ in range(steps):
        net.inject_current(p, np.array([0], np.uint32), np.array([100.0], np.float32))
        net.step(1)
        fired += net.spikes(p)
    return net, int(fired[1]), int(fired[2])


def lcg_net(seed, n, max_out=5, max_in=10):
    """The reference's Brain test connectome (P/api/learn/brain.rs:428-453):
    an LCG (Knuth's MMIX constants, >> 33) gives each source 0-4 synapses to
    random targets with weights in [0, 1); in-degree is capped at `max_in` so
    that a scripted network's synaptic input stays below threshold."""
    state = [seed]

    def nxt():
        state[0] = (state[0] * 6364136223846793005 + 1442695040888963407) & (2**64 - 1)
        return state[0] >> 33

    pre, post, w, indeg = [], [], [], np.zeros(n, np.int64)
    for src in range(n):
        for _ in range(nxt() % max_out):
            dst = nxt() % n
            wt = (nxt() % 1_000_000) / 1_000_000.0
            if indeg[dst] < max_in:
                indeg[dst] += 1
                pre.append(src)
                post.append(dst)
                w.append(wt)
    return np.array(pre, np.uint32), np.array(post, np.uint32), np.array(w, np.float32)


def learn_scripted(make_net, n, pre, post, w, spikes, cfg, actions=None, motor=None):
    """A network whose spikes are scripted: LIF neurons with dt = 1/tau = 1
    (v = v_rest + input each step, no refractory time) at rest 0, threshold
    50; a neuron fires when it is given 100 (the input clamp) through
    inject_current, and the synaptic input alone (in-degree <= 10, weights
    <= 4) stays below threshold.  Learning runs on the network's synapses;
    `actions[t]` (a list of (verb, args)) is applied after step t."""
    net = make_net()
    p = net.add_population(LIF, n)
    for col, v in enumerate([1.0, 1.0, 0.0, 50.0, 0.0, 0.0]):
        net.fill_param(p, col, v)
    net.connect(p, pre, p, post, w, np.ones(pre.size, np.uint8))
    net.build()
    net.enable_learning(**cfg)
    if motor is not None:
        net.set_motor(*motor)
    out = []
    for t, row in enumerate(spikes):
        idx = np.nonzero(row)[0].astype(np.uint32)
        if idx.size:
            net.inject_current(p, idx, np.full(idx.size, 100.0, np.float32))
        net.step(1)
        got = np.asarray(net.spikes(p))
        assert np.array_equal(got != 0, np.asarray(row) != 0), f"scripted spikes broke at step {t}"
        for verb, args in (actions or {}).get(t, []):
            r = getattr(net, verb)(*args)
            if r is not None:
                out.append((t, verb, r))
    return net, out


def learn_pool(make_net, creatures, cfg, steps):
    """Several scripted networks (creatures) as populations of one network,
    no synapses between them, learning on; creature k gets its own rewards
    (`acts[t]` = [(dopamine, gate)]) on its own CSR synapse range."""
    net = make_net()
    pops = []
    for n, pre, post, w, _, _ in creatures:
        p = net.add_population(LIF, n)
        for col, v in enumerate([1.0, 1.0, 0.0, 50.0, 0.0, 0.0]):
            net.fill_param(p, col, v)
        net.connect(p, pre, p, post, w, np.ones(pre.size, np.uint8))
        pops.append(p)
    net.build()
    net.enable_learning(**cfg)
    ranges = [net.population_synapses(p) for p in pops]
    for t in range(steps):
        for (n, _, _, _, spikes, _), p in zip(creatures, pops):
            idx = np.nonzero(spikes[t])[0].astype(np.uint32)
            if idx.size:
                net.inject_current(p, idx, np.full(idx.size, 100.0, np.float32))
        net.step(1)
        for k, ((n, _, _, _, spikes, acts), p) in enumerate(zip(creatures, pops)):
            assert np.array_equal(np.asarray(net.spikes(p)) != 0, spikes[t] != 0)
            for dop, gate in acts.get(t, []):
                net.reward(dop, gate, synapses=ranges[k])
    return net, pops, ranges


def pool_creatures(steps=300):
    out = []
    for seed, n, rate, every, phase, dop, gate in ((1, 24, 0.18, 10, 3, 1.0, 1.0), (2, 20, 0.25, 7, 2, -0.8, 0.5),
                                                   (3, 16, 0.12, 13, 5, 2.0, 0.75)):
        pre, post, w = lcg_net(seed, n)
        spikes = (np.random.default_rng(seed + 10).random((steps, n)) < rate).astype(np.int32)
        acts = {t: [(dop, gate)] for t in range(steps) if t % every == phase}
        out.append((n, pre, post, w, spikes, acts))
    return out
