"""The oracle against every golden vector the reference's own tests hold for
the simulation step (CPU only).  The pins are parsed from the reference test
files by tests/golden/make_reference_pins.py; each case cites its source."""
import numpy as np
import pytest

import oracle as O
import scenarios as S

PINS = S.PINS


def make_oracle():
    return O.Network(0)


@pytest.mark.parametrize("cfg", PINS["lif_spike_counts"]["configs"], ids=lambda c: c["label"])
def test_lif_golden_spike_counts(cfg):
    # tests/lif_vs_neuron.rs:77-140: mean count within 2 of 0 / 51 / 83
    pin = PINS["lif_spike_counts"]
    counts = S.lif_pin_counts(make_oracle, cfg, n=pin["n"], t_ms=pin["t_ms"], on_ms=pin["on_ms"])
    assert abs(counts.mean() - cfg["ref_spikes"]) <= pin["tolerance"]
    # the restatement is exact: every neuron gives the pinned count
    assert np.all(counts == int(cfg["ref_spikes"]))


@pytest.mark.parametrize("cfg", PINS["izh_patterns"]["configs"], ids=lambda c: c["label"])
def test_izhikevich_pattern_ranges(cfg):
    # tests/izhikevich_vs_neuron.rs:30-75,152-190
    per, cv = S.izh_pattern(make_oracle, cfg, PINS["izh_patterns"])
    avg = per.mean()
    assert cfg["min_spikes"] <= avg <= cfg["max_spikes"], avg
    assert cv >= cfg["min_isi_cv"]


@pytest.mark.parametrize("n", PINS["delay_arrival"]["sizes"])
def test_delay_arrival_exact(n):
    # tests/network_delays.rs:114-160: arrival exactly max(delay, 1) steps later
    delays = PINS["delay_arrival"]["delays"]
    d = [delays[i % len(delays)] for i in range(n)]
    a0, raster = S.delay_arrival(make_oracle, n, d)
    assert np.all(a0 == 1)
    for i, dl in enumerate(d):
        arrival = max(dl, 1)
        expect = np.zeros(raster.shape[0], np.int32)
        expect[arrival] = 1
        assert np.array_equal(raster[:, i], expect), (i, dl)
    assert raster.sum() == n


@pytest.mark.parametrize("case", PINS["push"]["cases"], ids=lambda c: c["name"])
def test_push_slot_arithmetic(case):
    # P/api/net/push.rs:300-499
    ring, spikes = S.push_case(make_oracle, case)
    assert sorted(np.nonzero(spikes)[0].tolist()) == sorted(case["active"])
    expect = np.zeros_like(ring)
    for slot, post, val in case["expect"]:
        expect[slot, post] += val
    assert np.array_equal(ring, expect)


def test_delay_ring_accumulate():
    # P/api/net/delay.rs:139-145: 3 + 4 accumulate to 7 in one cell
    case = dict(n=3, **{"from": [0, 1], "to": [2, 2]}, w=[3.0, 4.0], d=[2, 2], active=[0, 1], step=0)
    ring, _ = S.push_case(make_oracle, case)
    assert ring[2, 2] == 7.0


def test_compaction_pins():
    pin = PINS["compact"]
    s = [1 if i % pin["some"]["every"] == 0 else 0 for i in range(pin["some"]["n"])]
    assert O.compact(s).tolist() == pin["some"]["expect"]
    assert O.compact(pin["alternating"]["spikes"]).tolist() == pin["alternating"]["expect"]
    h = pin["hashed"]
    spikes = [1 if (i * h["mul"]) % (1 << 64) % h["mod"] < h["lt"] else 0 for i in range(h["n"])]
    out = O.compact(spikes)
    assert out.tolist() == [i for i, x in enumerate(spikes) if x]
    assert out.size >= h["min_len"]
    assert O.compact(np.zeros(100, np.int32)).size == 0
    assert O.compact(np.ones(64, np.int32)).tolist() == list(range(64))


def test_poisson_hash_properties():
    # P/api/net/network/sources.rs:5-14: deterministic, rate ~ p
    hits = sum(O.poisson_spike(7, 0, s, 0.2) for s in range(20000))
    assert abs(hits / 20000 - 0.2) < 0.01
    assert [O.poisson_spike(3, 0, s, 0.5) for s in range(50)] == [O.poisson_spike(3, 0, s, 0.5) for s in range(50)]
    assert not any(O.poisson_spike(1, 0, s, 0.0) for s in range(1000))
    assert all(O.poisson_spike(1, 0, s, 1.0) for s in range(1000))


def test_fast_exp_accuracy():
    # P/math/fast_exp.rs:20-22: rel. error < 0.001 for |x| < 80
    for x in np.linspace(-80, 80, 2001):
        assert abs(O.fast_exp(x) / np.exp(x) - 1) < 1e-3


def test_hh_exp_accuracy():
    for x in np.linspace(-80, 80, 4001, dtype=np.float32):
        e = np.exp(np.float64(x))
        assert abs(O.sg_expf(float(x)) / e - 1) < 4e-7


def test_contract_violations_raise():
    net = make_oracle()
    p = net.add_population(S.LIF, 4)
    with pytest.raises(O.OracleError):
        net.connect(p, [0], p, [9], [1.0], [0])  # to index out of bounds
    with pytest.raises(O.OracleError):
        net.connect(p, [0], p, [1], [1.0], [32])  # delay >= 32
    with pytest.raises(O.OracleError):
        net.connect(p, [0], p, [1], [float("nan")], [0])
    with pytest.raises(O.OracleError):
        net.step(1)  # before build
    net.build()
    with pytest.raises(O.OracleError):
        net.build()
    with pytest.raises(O.OracleError):
        net.connect(p, [0], p, [1], [1.0], [0])
    with pytest.raises(O.OracleError):
        net.inject_current(p, [4], [1.0])


def test_empty_network_advances_counter():
    # P/api/net/network/step.rs:22-25
    net = make_oracle()
    net.build()
    net.step(5)
    assert net.step_counter == 5


def test_izhikevich_pulse_network_activity():
    # the pulse-coupled network settles into the known ~5-10 Hz activity
    import simuse_b200.workloads as W
    spec = W.izhikevich_pulse(steps=300)
    net = make_oracle()
    pop = W.build_izhikevich(net, spec)
    idx = np.arange(spec["n"], dtype=np.uint32)
    tot = 0
    for t in range(300):
        net.inject_current(pop, idx, W.izhikevich_input(spec, t))
        net.step(1)
        tot += net.spikes(pop).sum()
    rate = tot / spec["n"] / 0.3
    assert 2.0 < rate < 20.0, rate


def test_fixed_indegree_generator_shape():
    import simuse_b200.workloads as W
    pre, post, w, d = W.fixed_indegree_edges(1000, 500, 50, 9, 800, 20.0, -100.0, 1, 20)
    assert pre.size == 500 * 50
    assert np.all(np.bincount(post, minlength=500) == 50)
    assert pre.max() < 1000 and d.min() >= 1 and d.max() <= 20
    assert np.all((w == 20.0) == (pre < 800))


def test_hh_fp32_vs_fp64_close():
    # HH-RK4 FP32 restatement stays close to its FP64 twin over 20 ms
    out = []
    for prec in (0, 1):
        net = O.Network(prec)
        p = net.add_population(S.HH, 16)
        for col, v in enumerate([0.01, 1.0, 120.0, 36.0, 0.3, 50.0, -77.0, -54.4, 10.0, 0.0]):
            net.fill_param(p, col, v)
        net.fill_state(p, 0, -65.0)
        net.fill_state(p, 1, 0.0529)
        net.fill_state(p, 2, 0.5961)
        net.fill_state(p, 3, 0.3177)
        net.build()
        r = net.step(2000, record=True)
        out.append((r, net.state_f64(p, 0)))
    (r32, v32), (r64, v64) = out
    assert np.array_equal(r32, r64)
    assert r32.sum() > 0
    assert np.max(np.abs(v32 - v64)) < 1e-2


def test_kuramoto_oracle_mean_field_is_the_dense_sum():
    """The oracle's mean-field coupling K*(S cos th_i - C sin th_i) equals the
    dense K/N sum_j sin(th_j - th_i) of P/kernels/phase/sparse.rs:40-140, and
    its RK4 + wrap (P/kernels/mod.rs:74-77) matches an independent FP64 RK4."""
    rng = np.random.default_rng(12)
    n, K, dt, steps = 48, 1.3, 0.05, 7
    th0 = rng.uniform(-np.pi, np.pi, n).astype(np.float32)
    om = rng.normal(0, 1, n).astype(np.float32)

    Kd, hd = float(np.float32(K)), float(np.float32(dt))  # the C ABI takes K and dt as f32

    def f(x):
        return om.astype(np.float64) + Kd / n * np.sin(x[None, :] - x[:, None]).sum(axis=1)

    x = th0.astype(np.float64)
    r_ref = []
    for _ in range(steps):
        k1 = f(x)
        k2 = f(x + hd / 2 * k1)
        k3 = f(x + hd / 2 * k2)
        k4 = f(x + hd * k3)
        x = x + hd / 6 * (k1 + 2 * k2 + 2 * k3 + k4)
        x = x - 2 * np.pi * np.round(x / (2 * np.pi))
        r_ref.append(abs(np.exp(1j * x).mean()))
    th, r = O.kuramoto_rk4(th0, om, K, dt, steps, precision=1)
    assert np.abs(np.angle(np.exp(1j * (th - x)))).max() < 1e-6  # th is rounded to f32
    assert np.abs(r - np.array(r_ref)).max() < 1e-12


def test_tm_matches_neuron_delivered_weights():
    """P/api/net/push.rs:646-695: delivered weights of a depressing and a
    facilitating Tsodyks-Markram synapse against NEURON, spikes at steps
    20 + 40k, dt 0.5 ms, within the reference's 1e-4."""
    pin = PINS["tm_neuron"]
    dt = np.float32(pin["dt"])
    dep, fac = pin["depression"], pin["facilitation"]
    a_dep = float(np.exp(np.float32(-dt / np.float32(dep["tau_rec"]))))
    got = O.tm_sequence(dep["u0"], a_dep, 0.0, False, pin["steps"])
    assert np.max(np.abs(got - np.array(dep["ref"], np.float32))) < pin["tol"]
    a_rec = float(np.exp(np.float32(-dt / np.float32(fac["tau_rec"]))))
    a_fac = float(np.exp(np.float32(-dt / np.float32(fac["tau_fac"]))))
    got = O.tm_sequence(fac["u0"], a_rec, a_fac, True, pin["steps"])
    assert np.max(np.abs(got - np.array(fac["ref"], np.float32))) < pin["tol"]


def test_tm_depressing_synapse_silences_its_post():
    """P/api/net/network/tests.rs:530-575: the static edge keeps driving its
    post, the depressed edge leaves its post silent."""
    _, static, plastic = S.tm_drive(lambda: O.Network(0))
    assert static > 20
    assert plastic == 0


def test_register_plasticity_rejects_invalid_profile():
    """P/api/net/network/tests.rs:577-593."""
    net = O.Network(0)
    for u0, tau in ((0.0, 1.0), (1.5, 1.0), (0.5, 0.0), (0.5, float("nan"))):
        with pytest.raises(O.OracleError):
            net.register_plasticity(u0, tau, 0.5)


def test_sg_logf_is_correctly_rounded():
    """The GPEA log (shared by the kernels and the oracle) equals the
    correctly rounded FP32 log on a strided sample of every float in
    [1e-12, 1e6] (the whole range was checked exhaustively once), and the
    usual special values."""
    import math
    lo = np.array([1e-12], np.float32).view(np.uint32)[0]
    hi = np.array([1e6], np.float32).view(np.uint32)[0]
    bits = np.arange(lo, hi, 2003, dtype=np.uint64).astype(np.uint32)
    xs = bits.view(np.float32)
    want = np.log(xs.astype(np.float64)).astype(np.float32)
    got = np.array([O.sg_logf(float(x)) for x in xs], np.float32)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert O.sg_logf(1.0) == 0.0
    assert O.sg_logf(0.0) == -math.inf
    assert math.isnan(O.sg_logf(-1.0))
    assert O.sg_logf(math.inf) == math.inf
    assert O.sg_logf(1e-40) == float(np.float32(math.log(np.float32(1e-40))))


def test_receptor_kinetics_known_answers():
    """The reference's receptor-kinetics tests
    (crates/SiMuse/crates/pillars/src/kernels/synapse/tests.rs) on the
    oracle's restatement of DecayFactors, decay_all and compute_currents,
    with the Mg-block values of the receptor.rs doc comment."""
    assert abs(O.receptor_factors(0.5)[0] - 0.7788) < 1e-3            # test_decay_factors_precision
    f = O.receptor_factors(2.0)                                          # test_decay_all_exponential
    assert abs(np.float32(1.0) * f[0] - 0.3679) < 1e-3
    assert abs(np.float32(2.0) * f[2] - 1.6375) < 1e-3
    g = np.zeros((7, 2), np.float32)                                     # test_compute_currents_ohmic_direction
    g[0, 0], g[2, 1] = 0.1, 0.2
    i = O.receptor_currents(g, [-65.0, -65.0])
    assert abs(i[0] - 6.5) < 0.01 and abs(i[1]) < 0.01
    v = np.array([-80.0, -65.0, -40.0, -20.0, 0.0, 20.0, 40.0], np.float32)   # test_nmda_mg_block_voltage_profile
    g = np.zeros((7, 7), np.float32)
    g[1] = 1.0
    i = O.receptor_currents(g, v)
    assert i[0] < 5.0 and abs(i[4]) < 1.0 and i[5] < -5.0
    g = np.zeros((7, 2), np.float32)                                     # test_gabab_and_machr_inhibitory
    g[3, 0], g[6, 1] = 1.0, 1.0
    i = O.receptor_currents(g, [-65.0, -65.0])
    assert abs(i[0] + 25.0) < 0.1 and abs(i[1] + 25.0) < 0.1
    n = 13                                                               # test_simd_tail_consistent
    k = np.arange(n, dtype=np.float32) + 1.0
    g = np.zeros((7, n), np.float32)
    g[0], g[1], g[2], g[4] = 0.1 * k, 0.05 * k, 0.02, 0.01
    v = -70.0 + np.arange(n, dtype=np.float32)
    i = O.receptor_currents(g, v)
    for idx in (0, 4, 12):
        b = O.nmda_mg_block(float(v[idx]))
        want = (0.1 * (idx + 1) * (0.0 - v[idx]) + 0.05 * (idx + 1) * b * (0.0 - v[idx])
                + 0.02 * (-65.0 - v[idx]) + 0.01 * (0.0 - v[idx]))
        assert abs(i[idx] - want) < 1e-4, idx
    # the formula 1 / (1 + 0.33 exp(-0.06 v)): 0.058 at rest (the doc comment
    # of receptor.rs rounds it to "0.02"), 0.95 at the spike peak
    for vv in (-65.0, 30.0, -200.0, 200.0):
        want = 1.0 / (1.0 + 0.33 * np.exp(np.clip(-0.06 * vv, -10, 10)))
        assert abs(O.nmda_mg_block(vv) - want) < 1e-5 * max(1.0, want), vv
    assert abs(O.nmda_mg_block(30.0) - 0.95) < 0.01


def test_receptor_types_from_nt_signs():
    """test_build_receptor_types_csr (kernels/synapse/tests.rs): rows of a
    +1 and a -1 neuron give AMPA, AMPA, GABA_A, GABA_A; the insect phenotype
    and the FlyWire table (pillars-connectome/src/data.rs:44-59, 465-523)."""
    from simuse_b200.synaptic import receptor_types_flywire, receptor_types_from_nt
    assert receptor_types_from_nt([0, 2, 4], [1.0, -1.0]).tolist() == [0, 0, 2, 2]
    assert receptor_types_from_nt([0, 2, 4], [1.0, -1.0], "insect").tolist() == [4, 4, 5, 5]
    assert receptor_types_from_nt([0, 1, 3], [-1.0]).tolist() == [2, 0, 0]     # missing NT: +1
    assert receptor_types_flywire([0, 1, 2, 3, 4, 5], [1.0, -1.0, 2.0, -2.0, 0.0]).tolist() == [4, 2, 5, 6, 2]


def test_receptor_network_step_order_on_the_oracle():
    """SynapticBrain::step on the oracle network: a spike at step t jumps
    its target's conductance, which is decayed once before it drives the
    target at step t + 1 (synaptic.rs:94-130)."""
    net = O.Network(0)
    net.set_receptor_kinetics(1.0)
    pop = net.add_population(2, 2)           # Izhikevich
    for col, v in enumerate((1.0, 0.02, 0.2, -65.0, 8.0, 0.0, 30.0)):
        net.fill_param(pop, col, v)
    net.fill_state(pop, 0, -65.0)
    net.fill_state(pop, 1, -13.0)
    net.connect(pop, [0], pop, [1], [0.5], [7], syn_types=[4])   # nAChR, delay ignored
    net.build()
    net.inject_current(pop, np.array([0], np.uint32), np.array([100.0], np.float32))
    net.step(1)
    assert net.spikes(pop).tolist() == [1, 0]
    g = net.receptor_conductances()
    assert g[4, 1] == np.float32(0.5) and np.count_nonzero(g) == 1
    net.step(1)
    assert net.spikes(pop)[0] == 0
    f = O.receptor_factors(1.0)
    assert net.receptor_conductances()[4, 1] == np.float32(0.5) * f[4]
