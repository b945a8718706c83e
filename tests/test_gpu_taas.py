""".taas v2 checkpoints of networks resident in HBM.

A built network saves its CSR synapses, weights, delays, synapse types and
(while learning) eligibility; the file must be the bytes the reference's
writer gives for the same sections (the oracle's restatement, fixed
`created`).  Resuming loads a snapshot's weights into a freshly built
network, which must then step as the oracle does with those weights; a
network can also be built from a snapshot's synapses.
"""
import numpy as np
import pytest

import oracle as O
import scenarios as S
import simuse_b200 as sg
import taas_oracle as T
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

CREATED = "2026-01-01T00:00:00Z"


def _u32(a):
    return np.asarray(a, np.float32).view(np.uint32)


def _random_lif(make_net, n=500, k=20, seed=6, connect=True):
    rng = np.random.default_rng(seed)
    net = make_net()
    p = net.add_population(S.LIF, n)
    for col, v in enumerate([0.5, 0.1, -70.0, -54.0, -70.0, 2.0]):
        net.fill_param(p, col, v)
    net.set_state(p, 0, rng.uniform(-70.0, -55.0, n).astype(np.float32))
    pre = np.repeat(np.arange(n, dtype=np.uint32), k)
    post = rng.integers(0, n, pre.size).astype(np.uint32)
    w = rng.uniform(-20.0, 40.0, pre.size).astype(np.float32)
    d = rng.integers(1, 9, pre.size).astype(np.uint8)
    if connect:
        net.connect(p, pre, p, post, w, d)
    return net, p


def _drive(net, p, steps, seed=2):
    rng = np.random.default_rng(seed)
    idx = np.arange(net.total_neurons, dtype=np.uint32)
    out = []
    for _ in range(steps):
        net.inject_current(p, idx, rng.uniform(0.0, 60.0, idx.size).astype(np.float32))
        net.step(1)
        out.append(np.asarray(net.spikes(p)).copy())
    return np.array(out)


def test_snapshot_bytes_match_the_reference_writer(tmp_path):
    n = 24
    pre, post, w = S.lcg_net(0xC0FFEE, n)
    spikes = (np.random.default_rng(1).random((120, n)) < 0.18).astype(np.int32)
    cfg = dict(dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=0.5, w_min=0.0, w_max=4.0)
    acts = {t: [("reward", (1.2,))] for t in range(7, 120, 12)}
    g, _ = S.learn_scripted(lambda: sg.Network(0), n, pre, post, w, spikes, cfg, acts)
    c, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, cfg, acts)
    p = tmp_path / "net.taas"
    g.save_taas(p, created=CREATED)
    rp, col, wc, d = c.graph()
    e, _, _, _ = c.learning_state()
    ref = T.to_bytes([("row_ptr", "i32", rp.astype(np.int32)), ("col_indices", "i32", col.astype(np.int32)),
                      ("values", "f32", wc), ("delays", "u8", d), ("syn_types", "u8", np.zeros(d.size, np.uint8)),
                      ("eligibility", "f32", e)],
                     metadata={"type": "Network", "n_neurons": str(n), "n_synapses": str(col.size), "step": "120"},
                     game="dioma", created=CREATED)
    assert p.read_bytes() == ref
    g.close()


def test_resume_from_a_checkpoint_steps_like_the_oracle(tmp_path):
    """Learn on a driven network, checkpoint, load the weights into a fresh
    network: it carries the learned weights and steps as the oracle does
    from the same weights."""
    def driven(make_net):
        net = make_net()
        spec = W.lif_balanced(n=2000, k_in=100, seed=3, ext_rate_hz=4000.0, ext_weight=100.0, w_exc=20.0, g=5.0)
        p = W.build_lif(net, spec, device_generator=isinstance(net, sg.Network))
        net.build()
        return net, p
    a, _ = driven(lambda: sg.Network(0))
    a.enable_learning(dt=0.1, tau_e=200.0, lr=2.0, w_min=-150.0, w_max=60.0)
    a.step(300)
    a.reward(1.0)
    a.step(100)
    a.reward(-0.5)
    path = tmp_path / "ckpt.taas"
    a.save_taas(path, zstd_level=3)
    sg.taas.validate(path)
    w_learned = a.weights()
    b, bp = driven(lambda: sg.Network(0))
    assert b.scatter_mode == "exact"
    b.load_weights_taas(path)
    assert b.scatter_mode == "ordered"
    assert np.array_equal(_u32(b.weights()), _u32(w_learned))
    c, cp = driven(lambda: O.Network(0))
    c.set_weights(sg.taas.read(path, "values", "f32"))
    b.enable_raster(400)
    b.step(400)
    rb = b.read_raster()
    rc = c.step(400, record=True)
    assert rb.sum() > 1000
    assert np.array_equal(rb, rc)
    assert np.array_equal(_u32(b.state(bp, 0)), _u32(c.state(cp, 0)))
    # a snapshot of other synapses is refused
    other, _ = _random_lif(lambda: sg.Network(0))
    other.build()
    with pytest.raises(sg.SimuseError, match="differ"):
        other.load_weights_taas(path)
    for x in (a, b, other):
        x.close()


def test_network_built_from_a_snapshot(tmp_path):
    a, ap = _random_lif(lambda: sg.Network(0))
    a.build()
    path = tmp_path / "a.taas"
    a.save_taas(path)
    b, bp = _random_lif(lambda: sg.Network(0), connect=False)
    b.connect_taas(bp, bp, path)
    b.build()
    for x, y in zip(a.graph(), b.graph()):
        assert np.array_equal(np.asarray(x).view(np.uint8), np.asarray(y).view(np.uint8))
    assert np.array_equal(_drive(a, ap, 200), _drive(b, bp, 200))
    # the reference's connectome sections (no delays): default delay
    n = 500
    rp, col, w, _ = a.graph()
    conn = tmp_path / "conn.taas"
    conn.write_bytes(T.to_bytes([("row_ptr", "i32", rp.astype(np.int32)), ("col_indices", "i32", col.astype(np.int32)),
                                 ("values", "f32", w), ("nt_types", "f32", np.zeros(w.size, np.float32))],
                                game="dioma"))
    c, cp = _random_lif(lambda: sg.Network(0), connect=False)
    c.connect_taas(cp, cp, conn, default_delay=3)
    c.build()
    assert np.all(c.graph()[3] == 3) and np.array_equal(c.graph()[1], col)
    with pytest.raises(sg.SimuseError, match="row_ptr length"):
        d = sg.Network(0)
        q = d.add_population(S.LIF, n + 1)
        d.connect_taas(q, q, conn)
    for x in (a, b, c):
        x.close()
