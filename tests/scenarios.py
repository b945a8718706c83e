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
