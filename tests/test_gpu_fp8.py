"""FP8 E4M3 weight storage with a per-row scale (FP32 accumulation, FP32 state).

Each CSR row keeps scale = max|w| * 2^-8 (a power-of-two factor, so the
row's largest weight decodes exactly) and one E4M3 byte per synapse, the
nearest E4M3 value of w / scale: 5 bytes per synapse instead of 8.  Rows
whose weights are equal (the balanced LIF network: 20 and -100) therefore
keep their exact weights and give the FP32 path's bits; random weights are
rounded to 3 mantissa bits, and the population firing rate stays within the
stated tolerance of the FP64 oracle run with the unrounded weights.
"""
import numpy as np
import pytest

import oracle as O
import scenarios as SC
import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu

RATE_TOL = 0.01   # relative population-rate error vs the FP64 oracle


def _e4m3_values():
    c = np.arange(127)                    # non-negative finite codes (0x7F is NaN)
    ex, m = c >> 3, c & 7
    return np.where(ex == 0, m * 2.0 ** -9, (1.0 + m / 8.0) * 2.0 ** (ex - 7))


def e4m3_round(x):
    """Nearest E4M3 value (ties to the even code, saturating at 448), FP32."""
    v = _e4m3_values()
    ax = np.abs(np.asarray(x, np.float64))
    i = np.clip(np.searchsorted(v, ax), 1, 126)
    lo, hi = v[i - 1], v[i]
    up = (ax - lo > hi - ax) | ((ax - lo == hi - ax) & (i % 2 == 0))
    r = np.where(up, hi, lo)
    r = np.where(ax >= 448.0, 448.0, np.where(ax == 0.0, 0.0, r))
    return (np.sign(x) * r).astype(np.float32)


def fp8_weights(row_ptr, w):
    """The decoded weights the device stores for FP32 weights `w` in CSR rows."""
    out = np.empty_like(w)
    for r in range(row_ptr.size - 1):
        a, b = int(row_ptr[r]), int(row_ptr[r + 1])
        if a == b:
            continue
        sc = np.float32(np.abs(w[a:b]).max()) * np.float32(2.0 ** -8)
        if sc == 0:
            out[a:b] = 0
            continue
        q = e4m3_round((w[a:b] / sc).astype(np.float32))
        out[a:b] = (q * sc).astype(np.float32)
    return out


def _fmt(fmt):
    def make():
        net = sg.Network(0)
        if fmt is not None:
            net.set_weight_format(fmt)
        return net
    return make


def test_fp8_row_uniform_weights_give_fp32_bits_and_smaller_footprint():
    a, pa, ra = SC.lif_small_balanced(_fmt(None), n=3000, k_in=200, steps=300, device_generator=True)
    b, pb, rb = SC.lif_small_balanced(_fmt(sg.W_FP8), n=3000, k_in=200, steps=300, device_generator=True)
    assert b.scatter_mode == "exact"   # 20, -100 and 100 stay exact: the pre-centric path
    assert ra.sum() > 1000
    assert np.array_equal(ra, rb)
    assert np.array_equal(a.state(pa, 0).view(np.uint32), b.state(pb, 0).view(np.uint32))
    saved = a.footprint - b.footprint
    assert saved >= 3 * a.num_synapses - 4 * a.total_neurons - 4096
    a.close()
    b.close()


def _izh_rates(make, n, seeds, steps):
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


def test_fp8_random_weights_rate_within_tolerance_of_fp64_oracle():
    n, seeds, steps = 1000, [31, 32, 33], 400
    t8, g8 = _izh_rates(_fmt(sg.W_FP8), n, seeds, steps)
    t64, _ = _izh_rates(lambda: O.Network(precision=1), n, seeds, steps)
    err8 = abs(t8 - t64) / t64
    print(f"spikes fp64 {t64} fp8 {t8} ({err8:.4f})")
    assert t64 > 1000
    assert err8 <= RATE_TOL
    # the stored weights are the per-row E4M3 rounding of the given ones
    rp, col, wg, d = g8.graph()
    pre, post, w = W.fixed_outdegree_edges(n, 100, seeds[0], n * 4 // 5, 0.5, -1.0)
    order = np.lexsort((post, pre))
    want = fp8_weights(rp[:n + 1], w[order])
    assert np.array_equal(wg[:w.size].view(np.uint32), want.view(np.uint32))
    assert g8.scatter_mode == "ordered"
    g8.close()


def test_fp8_refuses_stdp_and_learning():
    net = sg.Network(0)
    p = net.add_population(sg.LIF, 100)
    net.set_weight_format(sg.W_FP8)
    net.stdp_config(0.1, 20.0, 20.0, 0.01, 0.0105, 0.0, 1.0)
    net.connect(p, np.arange(100, dtype=np.uint32), p, np.arange(100, dtype=np.uint32)[::-1].copy(),
                np.full(100, 0.5, np.float32), np.ones(100, np.uint8), stdp=True)
    with pytest.raises(sg.SimuseError, match="STDP"):
        net.build()
    net.close()
    net = sg.Network(0)
    p = net.add_population(sg.LIF, 100)
    net.set_weight_format(sg.W_FP8)
    net.connect(p, np.arange(100, dtype=np.uint32), p, np.arange(100, dtype=np.uint32)[::-1].copy(),
                np.full(100, 0.5, np.float32), np.ones(100, np.uint8))
    net.build()
    with pytest.raises(sg.SimuseError, match="FP8"):
        net.enable_learning()
    net.close()


def test_e4m3_rounding_twin_matches_known_values():
    x = np.array([0, 1, 448, 500, 1.0625, 1.1875, 2 ** -9, 3 * 2 ** -10, -17.0, 240, 232], np.float32)
    want = np.array([0, 1, 448, 448, 1.0, 1.25, 2 ** -9, 2 ** -8, -16.0, 240, 224], np.float32)
    assert np.array_equal(e4m3_round(x), want)
