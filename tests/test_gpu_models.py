"""HH-RK4 with ExpOne conductance synapses and pair STDP, and GPEA, on the
GPU against the CPU oracle (FP32 twin; FP64 twin for accuracy statements)."""
import numpy as np
import pytest

import oracle as O
import scenarios as S

pytestmark = pytest.mark.gpu


def gpu():
    from simuse_b200 import Network
    return Network(0)


def test_hh_kinetics_stdp_bit_identical():
    g, (ge, gi), rg = S.hh_network(gpu)
    c, (ce, ci), rc = S.hh_network(lambda: O.Network(0))
    assert rc.sum() > 20, rc.sum()
    assert np.array_equal(rg, rc)
    for pg, pc in ((ge, ce), (gi, ci)):
        for col in range(4):
            assert np.array_equal(g.state(pg, col).view(np.uint32), c.state(pc, col).view(np.uint32)), col
    # plastic weights: every synapse updated by one thread per pass -> exact
    wg, wc = g.weights(), c.weights()
    assert np.array_equal(np.sort(wg), np.sort(wc))
    rp, col, w, d = g.graph()
    rpc, colc, wcc, dc = c.graph()
    assert np.array_equal(rp, rpc)
    # rows are stored sorted by target on the device: compare row multisets
    for i in range(rp.size - 1):
        a = sorted(zip(col[rp[i]:rp[i + 1]].tolist(), d[rp[i]:rp[i + 1]].tolist(), wg[rp[i]:rp[i + 1]].tolist()))
        b = sorted(zip(colc[rpc[i]:rpc[i + 1]].tolist(), dc[rpc[i]:rpc[i + 1]].tolist(), wc[rpc[i]:rpc[i + 1]].tolist()))
        assert a == b, i
    # FP64 drift accumulator: summation order differs, tolerance 1e-9 relative
    dg, dcpu = g.stdp_drift, c.stdp_drift
    assert dcpu != 0.0
    assert abs(dg - dcpu) <= 1e-9 * max(1.0, abs(dcpu))
    xg, yg = g.stdp_traces()
    xc, yc = c.traces()
    assert np.array_equal(xg, xc) and np.array_equal(yg, yc)
    # kinetic rings hold identical values
    for ring in (1, 2):
        assert np.array_equal(g.ring(ring).view(np.uint32), c.ring(ring).view(np.uint32))


def test_hh_fp32_close_to_fp64_twin():
    c32, (e32, _), r32 = S.hh_network(lambda: O.Network(0), steps=300)
    c64, (e64, _), r64 = S.hh_network(lambda: O.Network(1), steps=300)
    # chaotic dynamics: rasters agree up to the first divergence, which must
    # come late; membrane potentials stay close before it
    diff = np.nonzero((r32 != r64).any(axis=1))[0]
    first = diff[0] if diff.size else r32.shape[0]
    assert first >= 250, first


def test_gpea_bit_identical_to_oracle():
    """GPEA (exponential-Euler gates with the project's fast_exp, calcium
    Nernst potential with sg_logf, implicit-Euler membrane): states and
    rasters bit-identical to the oracle."""
    g, pg, rg = S.gpea_network(gpu)
    c, pc, rc = S.gpea_network(lambda: O.Network(0))
    assert rg.sum() > 0
    assert np.array_equal(rg, rc)
    for col in range(9):
        a, b = g.state(pg, col), c.state(pc, col)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (col, np.abs(a - b).max())


def test_empty_and_isolated_populations():
    for mk in (gpu, lambda: O.Network(0)):
        net = mk()
        a = net.add_population(S.LIF, 0)
        b = net.add_population(S.IZH, 3)
        net.build()
        net.step(3)
        assert net.spikes(a).size == 0
        assert net.step_counter == 3
