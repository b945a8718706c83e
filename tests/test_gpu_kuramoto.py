"""Batched Kuramoto RK4 on the GPU against the FP64 oracle.

The reference's phase kernels (crates/SiMuse/crates/pillars/src/kernels/phase/
kuramoto.rs:42-68, sparse.rs:40-140) integrate one population by forward
Euler; the batched RK4 form with the mean-field identity
(crates/SiMuse/crates/t3/src/oscillator.rs:15-20,549) has no reference
implementation, so parity is against the oracle's FP64 restatement:
r(t) within 1e-3 absolute at every recorded step, phases within a circular
distance of 1e-3 for the median oscillator.
"""
import numpy as np
import pytest

import oracle as O
from simuse_b200 import KuramotoBatch
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

R_TOL = 1e-3       # order parameter, absolute, every step
THETA_MED_TOL = 1e-3


def _circ(a, b):
    return np.abs(np.angle(np.exp(1j * (a.astype(np.float64) - b.astype(np.float64)))))


def _sweep(sizes, ks, seed=4):
    sizes = np.asarray(sizes, np.uint32)
    total = int(sizes.astype(np.int64).sum())
    j = np.arange(total, dtype=np.uint64)
    theta = ((W.uniform01(seed, 2, j) * 2 - 1) * np.pi).astype(np.float32)
    omega = (0.5 * np.tan(np.pi * (np.clip(W.uniform01(seed, 3, j), 1e-12, 1 - 1e-12) - 0.5))).astype(np.float32)
    return sizes, np.asarray(ks, np.float32), theta, omega


# sizes reach every kernel shape: resident CTAs of 64 (partial and full),
# 128, 256 and 512 threads; clusters of 2 (4097: one oscillator in the
# second CTA), 4, 8 CTAs of 512 threads (16384 and 32768 fill them) and
# 8 CTAs of 1024 threads up to the 65,536 maximum
SIZES = [256, 512, 1000, 2048, 4096, 4097, 9000, 20000, 65536, 16384, 32769]
KS = [0.0, 1.5, 0.7, 1.2, 1.5, 2.0, 2.5, 3.0, 4.0, 1.0, 3.5]


def test_kuramoto_batch_vs_fp64_oracle():
    steps, dt = 800, 0.01
    sizes, ks, th0, om = _sweep(SIZES, KS)
    kb = KuramotoBatch(sizes, ks, dt)
    kb.set_state(th0, om)
    kb.record(steps)
    kb.run(steps // 2)
    kb.run(steps - steps // 2)
    th = kb.theta()
    r = kb.r()
    rmean = kb.r_mean()
    assert r.shape == (len(SIZES), steps)
    off = np.concatenate([[0], np.cumsum(sizes.astype(np.int64))])
    for i, (n, k) in enumerate(zip(SIZES, KS)):
        o_th, o_r = O.kuramoto_rk4(th0[off[i]:off[i + 1]], om[off[i]:off[i + 1]], float(k), dt, steps, precision=1)
        dr = np.abs(r[i].astype(np.float64) - o_r).max()
        assert dr <= R_TOL, (n, k, dr)
        d = _circ(th[off[i]:off[i + 1]], o_th)
        assert np.median(d) <= THETA_MED_TOL, (n, k, np.median(d))
        assert abs(rmean[i] - o_r.mean()) <= R_TOL, (n, k, rmean[i], o_r.mean())
        # the FP64 time average is the mean of the recorded FP32 r(t)
        assert abs(rmean[i] - r[i].astype(np.float64).mean()) <= 1e-6
    kb.close()


def test_kuramoto_deterministic_and_alone_equals_batched():
    """Same inputs -> same bits; an instance alone gives the bits it gives
    inside a batch (the batch composition does not change the arithmetic)."""
    steps, dt = 300, 0.01
    sizes, ks, th0, om = _sweep(SIZES, KS, seed=9)
    runs = []
    for _ in range(2):
        kb = KuramotoBatch(sizes, ks, dt)
        kb.set_state(th0, om)
        kb.record(steps)
        kb.run(steps)
        runs.append((kb.theta(), kb.r()))
        kb.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    off = np.concatenate([[0], np.cumsum(sizes.astype(np.int64))])
    for i in (1, 4, 5, 6, 8, 10):
        kb = KuramotoBatch(sizes[i:i + 1], ks[i:i + 1], dt)
        kb.set_state(th0[off[i]:off[i + 1]], om[off[i]:off[i + 1]])
        kb.record(steps)
        kb.run(steps)
        assert np.array_equal(kb.theta(), runs[0][0][off[i]:off[i + 1]])
        assert np.array_equal(kb.r()[0], runs[0][1][i])
        kb.close()


def test_kuramoto_streamed_form_vs_fp64_oracle(monkeypatch):
    """The streamed form (one CTA per instance, state re-read every stage),
    which instances above 4096 oscillators take on a device that cannot hold
    their cluster shape, forced here through SG_KURAMOTO_STREAMED."""
    monkeypatch.setenv("SG_KURAMOTO_STREAMED", "1")
    steps, dt = 300, 0.01
    sizes, ks, th0, om = _sweep([5000, 40000], [2.0, 3.0], seed=5)
    kb = KuramotoBatch(sizes, ks, dt)
    kb.set_state(th0, om)
    kb.record(steps)
    kb.run(steps)
    r = kb.r()
    off = [0, 5000, 45000]
    for i in range(2):
        _, o_r = O.kuramoto_rk4(th0[off[i]:off[i + 1]], om[off[i]:off[i + 1]], float(ks[i]), dt, steps, precision=1)
        assert np.abs(r[i].astype(np.float64) - o_r).max() <= R_TOL
    kb.close()


def test_kuramoto_uncoupled_is_rotation():
    """K = 0: every phase rotates at its own frequency, r(t) of the batch
    instance equals |mean exp(i(theta0 + omega t))|."""
    steps, dt = 500, 0.01
    sizes, ks, th0, om = _sweep([3000], [0.0], seed=2)
    om = np.clip(om, -5, 5)
    kb = KuramotoBatch(sizes, ks, dt)
    kb.set_state(th0, om)
    kb.record(steps)
    kb.run(steps)
    th = kb.theta()
    exact = th0.astype(np.float64) + om.astype(np.float64) * steps * dt
    assert _circ(th, exact).max() <= 5e-4
    t = np.arange(1, steps + 1) * dt
    z = np.exp(1j * (th0[None, :].astype(np.float64) + om[None, :].astype(np.float64) * t[:, None]))
    r_exact = np.abs(z.mean(axis=1))
    assert np.abs(kb.r()[0] - r_exact).max() <= 1e-4
    kb.close()


def test_kuramoto_errors():
    from simuse_b200 import SimuseError
    with pytest.raises(SimuseError):
        KuramotoBatch([0], [1.0], 0.01)
    with pytest.raises(SimuseError):
        KuramotoBatch([70000], [1.0], 0.01)
    with pytest.raises(SimuseError):
        KuramotoBatch([10], [1.0], -0.01)
    kb = KuramotoBatch([10], [1.0], 0.01)
    with pytest.raises(SimuseError):
        kb.r()  # recording not enabled
    kb.record(5)
    kb.run(5)
    with pytest.raises(SimuseError):
        kb.run(1)  # record full
    assert kb.r().shape == (1, 5)
    kb.close()
