"""The uneven Kuramoto + Izhikevich sweep (simuse_b200.Sweep): both halves
run concurrently on one GPU.

* Every Izhikevich instance (BF16 weights 0.5 U / -U, U on the 1/256 grid,
  device thalamic noise) gives the FP32 oracle's spike counts and final
  membrane potentials bit for bit, and the sweep's total spike count is
  within RATE_TOL of the FP64 oracle's.
* Every Kuramoto instance's r(t) is within R_TOL of the FP64 oracle at every
  step, and its phases and r(t) are the bits the same batch gives alone.
* The autotuned scatter schedule gives the same bits as the fixed one.
"""
import numpy as np
import pytest

import oracle as O
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

RATE_TOL = 0.01   # relative, total spikes of the Izhikevich half vs the FP64 oracle
R_TOL = 1e-3      # Kuramoto order parameter, absolute, every step

IZH_STEPS, KURA_STEPS = 300, 800


def _oracle_instance(n, seed, steps, precision):
    """Spikes per neuron and final v of one sweep instance on the oracle,
    fed the thalamic input the device draws (host form)."""
    onet = O.Network(precision=precision)
    pop = W.add_izhikevich_instance(onet, n, seed, device_edges=False, device_noise=False, random_w=8)
    onet.build()
    idx = np.arange(n, dtype=np.uint32)
    counts = np.zeros(n, np.int64)
    for t in range(steps):
        onet.inject_current(pop, idx, W.thalamic_input(n, seed, t))
        onet.step(1)
        counts += onet.spikes(pop).astype(np.int64)
    return counts, onet.state(pop, 0)


def _small():
    kura = W.kuramoto_sweep(12, n_min=256, n_max=20000, seed=5)
    sizes = W.izh_sweep_sizes(10, n_min=500, n_max=4000, seed=9)
    return kura, sizes


def test_sweep_halves_match_their_oracles():
    kura, sizes = _small()
    assert kura["sizes"].max() > 4096 and kura["sizes"].min() <= 4096   # resident and streamed CTAs
    sw = sg.Sweep(kura, sizes, izh_seed0=300)
    assert sw.net.scatter_mode == "exact"
    sw.record_r(KURA_STEPS)
    # two overlapping enqueues per half, then one wait
    sw.enqueue(IZH_STEPS // 2, KURA_STEPS // 2)
    sw.enqueue(IZH_STEPS - IZH_STEPS // 2, KURA_STEPS - KURA_STEPS // 2)
    sw.synchronize()
    assert sw.izh_steps == IZH_STEPS and sw.kura_steps == KURA_STEPS

    tot_dev = tot64 = 0
    for i, (n, s) in enumerate(zip(sw.izh_sizes, sw.izh_seeds)):
        c32, v32 = _oracle_instance(int(n), int(s), IZH_STEPS, 0)
        c64, _ = _oracle_instance(int(n), int(s), IZH_STEPS, 1)
        got = sw.izh_counts(i)
        assert np.array_equal(got, c32), (i, int(got.sum()), int(c32.sum()))
        assert np.array_equal(sw.izh_state(i).view(np.uint32), v32.view(np.uint32)), i
        tot_dev += int(got.sum())
        tot64 += int(c64.sum())
    err = abs(tot_dev - tot64) / tot64
    print(f"izh spikes: device {tot_dev}, fp64 oracle {tot64}, rel err {err:.2e}")
    assert tot64 > 1000
    assert err <= RATE_TOL

    r = sw.kura_r()
    assert r.shape == (len(kura["sizes"]), KURA_STEPS)
    off = np.concatenate([[0], np.cumsum(kura["sizes"].astype(np.int64))])
    worst = 0.0
    for i in range(len(kura["sizes"])):
        th0 = kura["theta"][off[i]:off[i + 1]]
        om = kura["omega"][off[i]:off[i + 1]]
        _, o_r = O.kuramoto_rk4(th0, om, float(kura["coupling"][i]), kura["dt"], KURA_STEPS, precision=1)
        dr = float(np.abs(r[i].astype(np.float64) - o_r).max())
        worst = max(worst, dr)
        assert dr <= R_TOL, (i, int(kura["sizes"][i]), dr)
    print(f"kuramoto max |r - r_fp64| {worst:.2e}")

    # the Kuramoto half alone: the same bits
    kb = sg.KuramotoBatch(kura["sizes"], kura["coupling"], kura["dt"])
    kb.set_state(kura["theta"], kura["omega"])
    kb.record(KURA_STEPS)
    kb.run(KURA_STEPS)
    assert np.array_equal(kb.theta().view(np.uint32), sw.kb.theta().view(np.uint32))
    assert np.array_equal(kb.r().view(np.uint32), r.view(np.uint32))
    kb.close()
    sw.close()


def test_sweep_autotuned_schedule_gives_the_fixed_schedule_bits():
    kura, sizes = _small()
    runs, tuned_steps = [], 0
    for tune in (True, False):
        sw = sg.Sweep(kura, sizes, izh_seed0=300)
        if tune:
            res = sw.net.autotune(steps=10)      # 27 candidates x (10 warm-up + 10 timed) steps
            assert res["variant"] >= 0 and 1 <= res["blocks_per_sm"] <= 3
            tuned_steps = sw.net.step_counter
            assert tuned_steps == 27 * 20
        else:
            sw.run(tuned_steps, 0)               # the same steps on the fixed schedule
        sw.run(IZH_STEPS, 100)
        runs.append(([sw.izh_counts(i) for i in range(len(sizes))], sw.izh_state(len(sizes) - 1).copy(),
                     sw.events_total))
        sw.close()
    (ca, va, ea), (cb, vb, eb) = runs
    assert ea == eb
    assert all(np.array_equal(a, b) for a, b in zip(ca, cb))
    assert np.array_equal(va.view(np.uint32), vb.view(np.uint32))
