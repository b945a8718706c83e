"""Dopamine-modulated eligibility learning in the oracle (P/api/learn/brain.rs).

The oracle restates the reference's lazy Brain: traces decay by fma with the
step's spike, eligibility is touched only on spikes, with gaps decayed by
repeated multiplication and one trailing decay per step, and folded to now at
reward time.  The reference states that this is bit-identical to its dense
per-synapse formulation (pillars-wgpu/shaders/dopamine.wgsl:44-98, every
synapse every step: e = (e - ltd + ltp or e + ltp - ltd, by pre < post) * d_e);
here the dense form is written out in numpy and the oracle must give its bits.
The remaining tests are the reference's own Brain tests (brain.rs:546-699)
and the zero-delta rule of its weight update (P/kernels/dopamine/tests.rs:64-86).
"""
from fractions import Fraction

import numpy as np

import oracle as O
import scenarios as S

CFG = dict(dt=0.5, tau_pre=20.0, tau_post=20.0, tau_e=1000.0, a_ltp=0.1, a_ltd=0.12, lr=0.5, w_min=0.0, w_max=4.0)
f32 = np.float32


def fma32(a, b, c):
    """a*b + c rounded once to float32 (nearest, ties to even)."""
    x = Fraction(float(a)) * Fraction(float(b)) + Fraction(float(c))
    r = f32(float(x))
    cands = (np.nextafter(r, f32(-np.inf)), r, np.nextafter(r, f32(np.inf)))
    return min(cands, key=lambda y: (abs(Fraction(float(y)) - x), int(np.array(y, f32).view(np.uint32)) & 1))


class Dense:
    """The dense formulation over the network's CSR synapses."""

    def __init__(self, n, pre, post, w, cfg):
        self.pre, self.post, self.w = pre.astype(np.int64), post.astype(np.int64), w.astype(f32).copy()
        self.cfg = cfg
        self.tp = np.zeros(n, f32)
        self.tq = np.zeros(n, f32)
        self.e = np.zeros(pre.size, f32)
        self.dp = f32(O.fast_exp(f32(-cfg["dt"]) / f32(cfg["tau_pre"])))
        self.dq = f32(O.fast_exp(f32(-cfg["dt"]) / f32(cfg["tau_post"])))
        self.de = f32(O.fast_exp(f32(-cfg["dt"]) / f32(cfg["tau_e"])))

    def step(self, s):
        s = np.asarray(s) != 0
        self.tp = np.array([fma32(x, self.dp, f32(1.0 if k else 0.0)) for x, k in zip(self.tp, s)], f32)
        self.tq = np.array([fma32(x, self.dq, f32(1.0 if k else 0.0)) for x, k in zip(self.tq, s)], f32)
        ltp = np.where(s[self.post], f32(self.cfg["a_ltp"]) * self.tp[self.pre], f32(0.0)).astype(f32)
        ltd = np.where(s[self.pre], f32(self.cfg["a_ltd"]) * self.tq[self.post], f32(0.0)).astype(f32)
        e = np.where(self.pre < self.post, (self.e - ltd) + ltp, (self.e + ltp) - ltd).astype(f32)
        self.e = (e * self.de).astype(f32)

    def reward(self, dopamine, w_cap=None):
        lr_dopa = f32(self.cfg["lr"]) * f32(dopamine)
        delta = (lr_dopa * self.e).astype(f32)
        hi = f32(self.cfg["w_max"] if w_cap is None else w_cap)
        w = np.clip((self.w + delta).astype(f32), f32(self.cfg["w_min"]), hi)
        self.w = np.where(delta != 0, w, self.w).astype(f32)


def _spikes(seed, n, steps, rate):
    rng = np.random.default_rng(seed)
    return (rng.random((steps, n)) < rate).astype(np.int32)


def test_lazy_oracle_matches_the_dense_formulation_bit_for_bit():
    """brain.rs:469-533 (lazy_eligibility_matches_dense_dynamics): 24 neurons,
    600 steps at 18 % firing, reward 1.2 every 12 steps; weights and the
    folded eligibility after every reward are identical, not just close."""
    n, steps = 24, 600
    pre, post, w = S.lcg_net(0xC0FFEE, n)
    assert pre.size > 16
    spikes = _spikes(1, n, steps, 0.18)
    acts = {t: [("reward", (1.2,)), ("learning_state", ()), ("weights", ())] for t in range(steps) if t % 12 == 7}
    net, out = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, acts)
    fresh, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes[:0], CFG)
    rp, col, w_csr, _ = fresh.graph()  # the CSR synapses as built, before any reward
    pre_csr = np.repeat(np.arange(n), np.diff(rp.astype(np.int64)))
    dense = Dense(n, pre_csr, col, w_csr, CFG)
    it = iter(out)
    for t in range(steps):
        dense.step(spikes[t])
        if t % 12 == 7:
            dense.reward(1.2)
            _, _, (e, tp, tq, tt) = next(it)
            _, _, wl = next(it)
            assert tt == t + 1
            assert np.array_equal(tp, dense.tp) and np.array_equal(tq, dense.tq), t
            assert np.array_equal(e, dense.e), t
            assert np.array_equal(wl, dense.w), t
    assert np.any(dense.w != w_csr)


def test_reward_skips_zero_deltas():
    """P/kernels/dopamine/tests.rs:64-86: synapses with zero eligibility keep
    weights outside [w_min, w_max]; the one with e = 1 moves by lr * D * e."""
    pre = np.zeros(16, np.uint32)
    post = np.arange(16, dtype=np.uint32) % 4
    w = np.zeros(16, np.float32)
    w[0], w[1], w[2] = 22.0, -3.0, 0.5
    net = O.Network(0)
    p = net.add_population(S.LIF, 4)
    net.connect(p, pre, p, post, w, np.ones(16, np.uint8))
    net.build()
    net.enable_learning(**dict(CFG, lr=0.1, w_max=6.0))
    rp, col, wc, _ = net.graph()
    e = np.zeros(16, np.float32)
    k = int(np.nonzero(wc == np.float32(0.5))[0][0])
    e[k] = 1.0
    net.set_eligibility(e)
    net.reward(1.0)
    w1 = net.weights()
    assert w1[wc == 22.0][0] == 22.0 and w1[wc == -3.0][0] == -3.0
    assert w1[k] == np.float32(0.5) + np.float32(0.1)


def _burn(reward):
    pre, post, w = np.array([0], np.uint32), np.array([1], np.uint32), np.array([0.5], np.float32)
    cfg = dict(CFG, a_ltp=0.3, a_ltd=0.02)
    spikes = np.array([[1, 0], [0, 1]] * 200, np.int32)
    acts = {t: [("reward", reward)] for t in range(1, 400, 2)}
    net, _ = S.learn_scripted(lambda: O.Network(0), 2, pre, post, w, spikes, cfg, acts)
    return float(net.weights()[0])


def test_birth_burn_raises_weights_above_the_working_cap():
    """brain.rs:650-699: pre-then-post pairing with reward_capped(2, 64)
    passes the working cap 4; the same pairing with reward(2) stops at it."""
    assert _burn((2.0, 1.0, 64.0)) > 4.0
    assert _burn((2.0,)) <= 4.0


def test_gate_zero_and_steps_alone_leave_weights():
    """brain.rs:546-587: stepping moves traces only; a closed gate (0) moves
    nothing; open rewards move weights."""
    n = 16
    pre, post, w = S.lcg_net(7, n)
    spikes = _spikes(3, n, 200, 0.15)
    net, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes[:50], CFG)
    w0 = net.weights()
    net.reward(1.5, 0.0)
    assert np.array_equal(net.weights(), w0)
    net.reward(1.5)
    assert not np.array_equal(net.weights(), w0)


def test_snapshot_recall_restores():
    """brain.rs:589-622: recall(1.0) brings the snapshot back to 1e-6."""
    n = 16
    pre, post, w = S.lcg_net(11, n)
    spikes = np.ones((80, n), np.int32)
    acts = {0: [("snapshot", ())]}
    acts.update({t: acts.get(t, []) + [("reward", (1.5,))] for t in range(80)})
    net, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, acts)
    net2, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes[:1], CFG)
    base = net2.weights()
    assert np.any(np.abs(net.weights() - base) > 1e-3)
    net.recall(1.0)
    assert np.max(np.abs(net.weights() - base)) < 1e-6


def test_clear_restrict_and_motor_counts():
    n = 20
    pre, post, w = S.lcg_net(5, n)
    spikes = _spikes(9, n, 60, 0.3)
    acts = {29: [("clear_eligibility", ()), ("learning_state", ())],
            40: [("restrict_eligibility", (np.arange(pre.size) % 2,)), ("learning_state", ())]}
    net, out = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, acts, motor=((0, 5), (5, 20)))
    e_clear = out[0][2][0]
    assert not np.any(e_clear)
    e_restr = out[1][2][0]
    assert not np.any(e_restr[0::2]) and np.any(e_restr[1::2])  # keep = index % 2
    # one step call: the counts are its spikes in each range
    net.step(1)
    s = np.asarray(net.spikes(0)) != 0
    assert net.motor_counts() == (int(s[:5].sum()), int(s[5:].sum()))


def test_learning_is_deterministic():
    """brain.rs:624-648."""
    n = 16
    pre, post, w = S.lcg_net(99, n)
    spikes = _spikes(0xDEAD, n, 200, 0.2)
    acts = {t: [("reward", (1.0,))] for t in range(0, 200, 5)}
    a, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, acts)
    b, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, acts)
    assert np.array_equal(a.weights(), b.weights())


def test_per_network_reward_in_a_pool_equals_separate_networks():
    """Three scripted networks as populations of one network, each rewarded on
    its own synapse range at its own times, end with the weights and
    eligibility each would have alone: the per-block reward the reference's
    pool lacks (dioma-engine/src/brain/dynamics/gpu_pool.rs:12-16)."""
    steps = 300
    cr = S.pool_creatures(steps)
    pool, pops, ranges = S.learn_pool(lambda: O.Network(0), cr, CFG, steps)
    w0 = S.learn_pool(lambda: O.Network(0), cr, CFG, 0)[0].weights()   # as built
    wp = pool.weights()
    ep = pool.learning_state()[0]
    for (n, pre, post, w, spikes, acts), (lo, hi) in zip(cr, ranges):
        a = {t: [("reward", x) for x in v] for t, v in acts.items()}
        alone, _ = S.learn_scripted(lambda: O.Network(0), n, pre, post, w, spikes, CFG, a)
        assert hi - lo == pre.size
        assert np.array_equal(wp[lo:hi], alone.weights())
        assert np.array_equal(ep[lo:hi], alone.learning_state()[0])
        assert np.count_nonzero(wp[lo:hi] != w0[lo:hi]) > 0        # each network learned
