"""BrainRunner on the GPU against the reference's run() semantics restated
with the oracle: a fresh Network per run() (runner.rs:1342-1440, brain.rs:
52-83) with the weights signed by nt_types, delay 0, the external current
injected into every step, v / u / refractory carried between calls."""
import numpy as np
import pytest

import oracle as O
from simuse_b200 import runner as R

pytestmark = pytest.mark.gpu


def _connectome(n=600, k=25, seed=4, w_hi=30.0):
    rng = np.random.default_rng(seed)
    row_ptr = np.arange(0, (n + 1) * k, k, dtype=np.int32)
    col = rng.integers(0, n, n * k).astype(np.int32)
    val = rng.uniform(0.0, w_hi, n * k).astype(np.float32)
    nt = np.where(rng.uniform(size=n) < 0.2, -1.0, 1.0).astype(np.float32)
    return R.ConnectomeData(row_ptr, col, val, nt)


class _ReferenceRunner:
    """The reference's current-based run() through the oracle."""

    def __init__(self, conn, cfg):
        self.conn, self.cfg, self.n = conn, cfg, conn.n_neurons
        self.lif = cfg.model == "lif"
        self.v = np.full(self.n, -58.0 if self.lif else -65.0, np.float32)
        self.u = np.full(self.n, -13.0, np.float32)
        self.refr = np.zeros(self.n, np.float32)

    def run(self, n_steps, ext):
        c, n = self.cfg, self.n
        net = O.Network()
        p = net.add_population(1 if self.lif else 2, n)
        if self.lif:
            cols = [c.dt_ms, np.float32(1.0) / np.float32(c.tau_m), c.v_rest, c.v_thresh, c.v_reset, c.tau_ref]
        else:
            cols = [c.dt_ms, c.a, c.b, c.c, c.d, c.tau_ref, 30.0]
        for k, v in enumerate(cols):
            net.fill_param(p, k, float(np.float32(v)))
        net.set_state(p, 0, self.v)
        if self.lif:
            net.set_state(p, 1, self.refr)
        else:
            net.set_state(p, 1, self.u)
            net.set_state(p, 2, self.refr)
        rp = self.conn.row_ptr.astype(np.int64)
        sign = np.where(self.conn.nt_types < 0, np.float32(-1.0), np.float32(1.0))
        pre = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp))
        w = self.conn.values * np.repeat(sign, np.diff(rp))
        net.connect(p, pre, p, self.conn.col_indices.astype(np.uint32), w.astype(np.float32),
                    np.zeros(pre.size, np.uint8))
        net.build()
        e = np.zeros(n, np.float32)
        ee = np.asarray(ext, np.float32)[:n]
        e[:ee.size] = ee
        idx = np.arange(n, dtype=np.uint32)
        out = np.zeros((n_steps, n), np.int32)
        for t in range(n_steps):
            net.inject_current(p, idx, e)
            net.step(1)
            out[t] = net.spikes(p)
        self.v = net.state(p, 0)
        if self.lif:
            self.refr = net.state(p, 1)
        else:
            self.u, self.refr = net.state(p, 1), net.state(p, 2)
        return out.reshape(-1)


@pytest.mark.parametrize("model", ["lif", "izh"])
def test_brain_runner_matches_reference_run_semantics(model):
    cfg = R.lif(0.1) if model == "lif" else R.izh(0.5)
    conn = _connectome(w_hi=30.0 if model == "lif" else 6.0)
    n = conn.n_neurons
    rng = np.random.default_rng(9)
    ext1 = rng.uniform(10.0, 16.0, n).astype(np.float32) if model == "lif" else rng.uniform(0, 12, n).astype(np.float32)
    ext2 = ext1[: n // 2] * np.float32(1.1)          # shorter than n: zeros past its end
    gpu, ref = R.BrainRunner(conn, cfg), _ReferenceRunner(conn, cfg)
    total = 0
    for steps, ext in ((150, ext1), (60, ext2), (1, ext1), (200, ext1)):
        a = gpu.run(steps, ext).copy()
        b = ref.run(steps, ext)
        total += a.sum()
        assert a.shape == (steps * n,)
        assert np.array_equal(a, b), (model, steps)
        assert np.array_equal(gpu.get_v(), ref.v)
        if model == "izh":
            assert np.array_equal(gpu.get_u(), ref.u)
    assert total > 100
    assert gpu.step_counter() == 411
    # firing_rates over the grow-only buffer (runner.rs:1002-1021)
    buf = gpu.spike_buffer
    n_steps = buf.size // n
    expect = (buf[:n_steps * n].reshape(n_steps, n) != 0).sum(0).astype(np.float32) / (
        np.float32(n_steps) * np.float32(cfg.dt_ms) / np.float32(1000.0))
    assert np.array_equal(gpu.firing_rates(cfg.dt_ms), expect)
    gpu.close()


def test_brain_runner_state_io_reset_and_errors():
    conn = _connectome(n=300)
    r = R.BrainRunner(conn, R.izh(0.5))
    v = np.linspace(-70, -60, 300).astype(np.float32)
    r.set_v(v)
    assert np.array_equal(r.get_v(), v)
    r.set_u(np.full(300, -12.0, np.float32))
    assert np.all(r.get_u() == -12.0)
    r.run(20, np.full(300, 8.0, np.float32))
    r.reset()
    i = np.arange(300, dtype=np.float32)
    expect = np.float32(-65.0) + ((i * np.float32(0.577)) % np.float32(1.0) - np.float32(0.5)) * np.float32(2.0) * np.float32(0.03)
    assert np.allclose(r.get_v(), expect, atol=1e-6) and r.step_counter() == 0
    r.add_poisson_group(np.arange(50), 400.0, 20.0)   # statistical drive (host RNG)
    s = r.run(200).reshape(200, 300)
    assert s[:, :50].sum() > s[:, 50:].sum() / 5
    r.close()
    with pytest.raises(ValueError, match="0 neurons"):
        R.BrainRunner(R.ConnectomeData(np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)), R.lif(0.1))
    bad = R.ConnectomeData(np.array([0, 1, 2], np.int32), np.array([1, 0], np.int32), np.array([1.0], np.float32))
    with pytest.raises(ValueError, match="col_indices length"):
        R.BrainRunner(bad, R.lif(0.1))


class _ReferenceSynapticRunner:
    """The reference's conductance run() (runner.rs:1365-1401, :1695-1735)
    through the oracle: a fresh SynapticBrain per call from the unsigned
    connectome and its receptor types, the last call's kinetics restored,
    state carried."""

    def __init__(self, conn, cfg, receptor_types):
        self.conn, self.cfg, self.n, self.rt = conn, cfg, conn.n_neurons, receptor_types
        self.lif = cfg.model.startswith("lif")
        self.v = np.full(self.n, -58.0 if self.lif else -65.0, np.float32)
        self.u = np.full(self.n, -13.0, np.float32)
        self.refr = np.zeros(self.n, np.float32)
        self.kin = None

    def run(self, n_steps, ext):
        c, n = self.cfg, self.n
        net = O.Network()
        net.set_receptor_kinetics(c.dt_ms)
        p = net.add_population(1 if self.lif else 2, n)
        if self.lif:
            cols = [c.dt_ms, np.float32(1.0) / np.float32(c.tau_m), c.v_rest, c.v_thresh, c.v_reset, c.tau_ref]
        else:
            cols = [c.dt_ms, c.a, c.b, c.c, c.d, c.tau_ref, 30.0]
        for k, v in enumerate(cols):
            net.fill_param(p, k, float(np.float32(v)))
        net.set_state(p, 0, self.v)
        if self.lif:
            net.set_state(p, 1, self.refr)
        else:
            net.set_state(p, 1, self.u)
            net.set_state(p, 2, self.refr)
        rp = self.conn.row_ptr.astype(np.int64)
        pre = np.repeat(np.arange(n, dtype=np.uint32), np.diff(rp))
        net.connect(p, pre, p, self.conn.col_indices.astype(np.uint32), self.conn.values.astype(np.float32),
                    np.ones(pre.size, np.uint8), syn_types=self.rt)
        net.build()
        if self.kin is not None:
            net.set_receptor_conductances(self.kin)
        e = np.zeros(n, np.float32)
        ee = np.asarray(ext, np.float32)[:n]
        e[:ee.size] = ee
        idx = np.arange(n, dtype=np.uint32)
        out = np.zeros((n_steps, n), np.int32)
        for t in range(n_steps):
            net.inject_current(p, idx, e)
            net.step(1)
            out[t] = net.spikes(p)
        self.kin = net.receptor_conductances()
        self.v = net.state(p, 0)
        if self.lif:
            self.refr = net.state(p, 1)
        else:
            self.u, self.refr = net.state(p, 1), net.state(p, 2)
        return out.reshape(-1)


@pytest.mark.parametrize("model", ["lif_synaptic", "izh_synaptic"])
def test_brain_runner_conductance_configs_match_reference(model):
    """LifSynaptic / IzhSynaptic: receptor types from the NT signs (AMPA /
    GABA_A), conductances carried across calls and cleared by reset."""
    cfg = R.lif_synaptic(0.1) if model == "lif_synaptic" else R.izh_synaptic(0.5)
    conn = _connectome(w_hi=0.05 if model == "lif_synaptic" else 0.02)
    n = conn.n_neurons
    from simuse_b200.synaptic import receptor_types_from_nt
    rt = receptor_types_from_nt(conn.row_ptr, conn.nt_types)
    assert set(np.unique(rt)) == {0, 2}
    rng = np.random.default_rng(3)
    ext1 = rng.uniform(14.0, 20.0, n).astype(np.float32) if model == "lif_synaptic" else \
        rng.uniform(0, 12, n).astype(np.float32)
    gpu, ref = R.BrainRunner(conn, cfg), _ReferenceSynapticRunner(conn, cfg, rt)
    total = 0
    for steps, ext in ((150, ext1), (60, ext1[: n // 2]), (1, ext1), (200, ext1)):
        a = gpu.run(steps, ext).copy()
        b = ref.run(steps, ext)
        total += a.sum()
        assert np.array_equal(a, b), (model, steps)
        assert np.array_equal(gpu.get_v().view(np.uint32), ref.v.view(np.uint32))
        assert np.array_equal(gpu.kinetics().view(np.uint32), ref.kin.view(np.uint32))
    assert total > 100
    assert np.count_nonzero(gpu.kinetics()) > 0
    gpu.reset()
    assert np.count_nonzero(gpu.kinetics()) == 0
    gpu.close()
