"""BF16 weight storage (FP32 accumulation, FP32 state).

Weights exactly representable in bf16 give the FP32 path's bits; random
weights are rounded to bf16 (relative error <= 2^-9), and the population
firing rate stays within the stated tolerance of the FP64 oracle run with
the unrounded weights."""
import numpy as np
import pytest

import oracle as O
import scenarios as SC
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

RATE_TOL = 0.01   # relative population-rate error vs the FP64 oracle (measured: 3e-4)


def _bf16(x):
    b = np.asarray(x, np.float32).view(np.uint32)
    r = ((b + np.uint32(0x7FFF) + ((b >> np.uint32(16)) & np.uint32(1))) >> np.uint32(16)) << np.uint32(16)
    return r.astype(np.uint32).view(np.float32)


def _lif(fmt):
    def make():
        net = sg.Network(0)
        if fmt is not None:
            net.set_weight_format(fmt)
        return net
    return make


def test_bf16_exact_weights_give_fp32_bits_and_smaller_footprint():
    a, pa, ra = SC.lif_small_balanced(_lif(None), n=3000, k_in=200, steps=300, device_generator=True)
    b, pb, rb = SC.lif_small_balanced(_lif(sg.W_BF16), n=3000, k_in=200, steps=300, device_generator=True)
    assert ra.sum() > 1000
    assert np.array_equal(ra, rb)
    assert np.array_equal(a.state(pa, 0), b.state(pb, 0))
    saved = a.footprint - b.footprint
    assert saved >= 2 * a.num_synapses - 4096
    a.close()
    b.close()


def _izh_rates(make, n, seeds, steps, precision=None):
    net = make()
    pops = [W.add_izhikevich_instance(net, n, s, device_edges=False, device_noise=False) for s in seeds]
    net.build()
    idx = np.arange(n, dtype=np.uint32)
    total = 0
    for t in range(steps):
        for p, s in zip(pops, seeds):
            net.inject_current(p, idx, W.thalamic_input(n, s, t))
        net.step(1)
        total += sum(int(net.spikes(p).sum()) for p in pops)
    return total, net


def test_bf16_random_weights_rate_within_tolerance_of_fp64_oracle():
    n, seeds, steps = 1000, [31, 32, 33], 400
    t16, g16 = _izh_rates(_lif(sg.W_BF16), n, seeds, steps)
    t32, g32 = _izh_rates(_lif(None), n, seeds, steps)
    t64, _ = _izh_rates(lambda: O.Network(precision=1), n, seeds, steps)
    err16, err32 = abs(t16 - t64) / t64, abs(t32 - t64) / t64
    print(f"spikes fp64 {t64} fp32 {t32} ({err32:.4f}) bf16 {t16} ({err16:.4f})")
    assert t64 > 1000
    assert err16 <= RATE_TOL and err32 <= RATE_TOL
    # the stored weights are the bf16 rounding of the given ones
    pre, post, w = W.fixed_outdegree_edges(n, 100, seeds[0], n * 4 // 5, 0.5, -1.0)
    rp, col, wg, d = g16.graph()
    order = np.lexsort((post, pre))
    assert np.array_equal(wg[:w.size], _bf16(w[order]))
    g16.close()
    g32.close()


def test_bf16_refuses_stdp():
    net = sg.Network(0)
    p = net.add_population(sg.LIF, 100)
    net.set_weight_format(sg.W_BF16)
    net.stdp_config(0.1, 20.0, 20.0, 0.01, 0.0105, 0.0, 1.0)
    net.connect(p, np.arange(100, dtype=np.uint32), p, np.arange(100, dtype=np.uint32)[::-1].copy(),
                np.full(100, 0.5, np.float32), np.ones(100, np.uint8), stdp=True)
    with pytest.raises(sg.SimuseError, match="STDP"):
        net.build()
    net.close()
