"""Receptor kinetics (SynapticBrain, crates/SiMuse/crates/pillars-connectome/
src/synaptic.rs:23-130) on the GPU against the FP32 oracle: spikes at every
step, final membrane potentials and all seven conductance arrays bit for
bit, for Izhikevich (four neurons per thread), LIF and HH (one per thread),
with every receptor code, codes >= 7 (AMPA), repeated (pre, post) synapses
and conductances carried across a kinetics write."""
import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg
from simuse_b200 import workloads as W
from simuse_b200.synaptic import SynapticBrain, receptor_types_from_nt

pytestmark = pytest.mark.gpu


def _graph(n, k, seed, w_exc, w_inh):
    """Fixed out-degree edges, each with a receptor code drawn by class
    (excitatory sources: AMPA, NMDA, nAChR or 9 (AMPA); inhibitory: GABA_A,
    GABA_B, GluCl, mAChR), plus repeated copies of some edges."""
    n_exc = n * 4 // 5
    pre, post, w = W.fixed_outdegree_edges(n, k, seed, n_exc, w_exc, w_inh)
    rng = np.random.default_rng(seed)
    exc = pre < n_exc
    rt = np.where(exc, rng.choice([0, 1, 4, 9], pre.size), rng.choice([2, 3, 5, 6], pre.size)).astype(np.uint8)
    dup = rng.choice(pre.size, pre.size // 50, replace=False)
    pre = np.concatenate([pre, pre[dup]])
    post = np.concatenate([post, post[dup]])
    w = np.concatenate([w, (w[dup] * np.float32(0.5)).astype(np.float32)])
    rt = np.concatenate([rt, rt[dup]])
    return pre.astype(np.uint32), post.astype(np.uint32), np.abs(w).astype(np.float32), rt


MEAN_LIF, MEAN_HH = 25.0, 9.0   # mean input: LIF v settles at its input (threshold 20); HH fires above ~7


def _izh(net, n, seed):
    a, b, c, d = W.izhikevich_params(n, n * 4 // 5, seed)
    pop = net.add_population(sg.IZH, n)
    net.fill_param(pop, 0, 1.0)
    for col, v in ((1, a), (2, b), (3, c), (4, d)):
        net.set_param(pop, col, v)
    net.fill_param(pop, 5, 0.0)
    net.fill_param(pop, 6, 30.0)
    net.fill_state(pop, 0, -65.0)
    net.set_state(pop, 1, (b * np.float32(-65.0)).astype(np.float32))
    return pop


def _lif(net, n, seed):
    pop = net.add_population(sg.LIF, n)
    for col, v in enumerate(W.LIF_PARAMS):
        net.fill_param(pop, col, v)
    u = W.uniform01(seed, W.LIF_STREAM_V0, np.arange(n, dtype=np.uint64))
    net.set_state(pop, 0, (10.0 + 10.0 * u).astype(np.float32))
    return pop


def _hh(net, n, seed):
    pop = net.add_population(sg.HH, n)
    for col, v in enumerate(W.HH_PARAMS):
        net.fill_param(pop, col, v)
    net.fill_state(pop, 0, -65.0)
    net.fill_state(pop, 1, 0.05)
    net.fill_state(pop, 2, 0.6)
    net.fill_state(pop, 3, 0.32)
    return pop


CASES = {
    # model builder, n, out-degree, weights (exc, inh), receptor dt, steps,
    # input mean, input sigma (exc, inh)
    "izh": (_izh, 3000, 60, 0.02, 0.04, 1.0, 400, 0.0, 5.0, 2.0),
    "lif": (_lif, 2000, 50, 0.002, 0.004, 0.1, 400, MEAN_LIF, 10.0, 10.0),
    "hh": (_hh, 400, 20, 0.004, 0.006, 0.01, 3000, MEAN_HH, 3.0, 3.0),
}


def _run(make_net, case, write_at=None):
    build, n, k, we, wi, dt, steps, mu, s_e, s_i = CASES[case]
    net = make_net()
    net.set_receptor_kinetics(dt)
    pop = build(net, n, 11)
    pre, post, w, rt = _graph(n, k, 11, we, wi)
    net.connect(pop, pre, pop, post, w, np.full(w.size, 3, np.uint8), syn_types=rt)
    net.build()
    idx = np.arange(n, dtype=np.uint32)
    sig = np.where(idx < n * 4 // 5, s_e, s_i)
    raster = np.zeros((steps, n), np.uint8)
    for t in range(steps):
        z = W.std_normal(77, 3, np.arange(n, dtype=np.uint64) + np.uint64(t * n))
        net.inject_current(pop, idx, (mu + sig * z).astype(np.float32))
        if write_at is not None and t == write_at:
            g = net.receptor_conductances()
            net.set_receptor_conductances((g * np.float32(0.5)).astype(np.float32))
        net.step(1)
        raster[t] = net.spikes(pop) != 0
    return raster, net.state(pop, 0).copy(), net.receptor_conductances(), net


@pytest.mark.parametrize("case", list(CASES))
def test_receptor_kinetics_bit_identical_to_oracle(case):
    rg, vg, gg, g = _run(lambda: sg.Network(0), case, write_at=CASES[case][6] // 2)
    ro, vo, go, _ = _run(lambda: O.Network(0), case, write_at=CASES[case][6] // 2)
    assert g.scatter_mode == "ordered"
    assert rg.sum() > 200, rg.sum()
    diff = np.nonzero((rg != ro).any(axis=1))[0]
    assert diff.size == 0, f"first divergent step {diff[0]}"
    assert np.array_equal(vg.view(np.uint32), vo.view(np.uint32))
    assert np.array_equal(gg.view(np.uint32), go.view(np.uint32))
    assert np.count_nonzero(gg) > 0
    g.close()


def test_synaptic_brain_facade_matches_network_form():
    """SynapticBrain.from_connectome (receptor types from NT signs) steps as
    the same network through the Network API."""
    n, k = 1500, 40
    pre, post, w, _ = _graph(n, k, 5, 0.02, 0.04)
    order = np.lexsort((post, pre))
    pre, post, w = pre[order], post[order], w[order]
    row_ptr = np.concatenate([[0], np.cumsum(np.bincount(pre, minlength=n))]).astype(np.uint32)
    nt = np.where(np.arange(n) < n * 4 // 5, 1.0, -1.0).astype(np.float32)
    brain = SynapticBrain.from_connectome(sg.IZH, row_ptr, post, w, 1.0, nt_types=nt)
    ref = O.Network(0)
    ref.set_receptor_kinetics(1.0)
    rp = _izh(ref, n, 5)
    ref.connect(rp, pre, rp, post, w, np.ones(w.size, np.uint8), syn_types=receptor_types_from_nt(row_ptr, nt))
    ref.build()

    def cfg(b):
        a, bb, c, d = W.izhikevich_params(n, n * 4 // 5, 5)
        b.fill_param(0, 1.0)
        for col, v in ((1, a), (2, bb), (3, c), (4, d)):
            b.set_param(col, v)
        b.fill_param(5, 0.0)
        b.fill_param(6, 30.0)
        b.fill_state(0, -65.0)
        b.set_state(1, (bb * np.float32(-65.0)).astype(np.float32))
    brain.configure(cfg)
    idx = np.arange(n, dtype=np.uint32)
    total = 0
    for t in range(300):
        ext = W.thalamic_input(n, 5, t)
        s = brain.step(ext)
        ref.inject_current(rp, idx, ext)
        ref.step(1)
        assert np.array_equal(s, ref.spikes(rp).astype(np.int32)), t
        total += int(s.sum())
    assert total > 100
    assert np.array_equal(brain.kinetics().view(np.uint32), ref.receptor_conductances().view(np.uint32))
    assert np.array_equal(brain.state(0).view(np.uint32), ref.state(rp, 0).view(np.uint32))
    assert len(brain) == n
    brain.close()


def test_receptor_mode_refusals():
    net = sg.Network(0)
    pop = net.add_population(sg.IZH, 100)
    net.connect(pop, [0], pop, [1], [0.1], [1])
    with pytest.raises(sg.SimuseError, match="before any synapse"):
        net.set_receptor_kinetics(1.0)
    net.close()
    net = sg.Network(0)
    net.set_receptor_kinetics(1.0)
    pop = net.add_population(sg.IZH, 100)
    with pytest.raises(sg.SimuseError, match="Poisson"):
        net.add_poisson_source(10.0, 1.0, 3)
    with pytest.raises(sg.SimuseError, match="kinetic profiles"):
        net.register_expone(5.0, 0.0, 1.0)
    with pytest.raises(sg.SimuseError, match="STDP"):
        net.connect(pop, [0], pop, [1], [0.1], [1], stdp=True)
    net.connect(pop, [0, 1], pop, [1, 2], [0.1, 0.2], [1, 1], syn_types=[1, 200])
    net.build()
    st, _ = net.graph_types()
    assert st.tolist() == [1, 0]                      # 200 is AMPA
    pool = sg.Pool(0)
    with pytest.raises(sg.SimuseError, match="pre-centric"):
        pool.add(net)
    pool.close()
    with pytest.raises(sg.SimuseError, match="conductances"):
        net.ring(0)
    net.close()
