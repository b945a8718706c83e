"""Failure detection without a GPU fault: every wait of the scatter pipeline
(its producer filling shared-memory stages with bulk copies, its consumers
issuing the reds) gives up after about a second, records the failure in a
device error word and leaves the kernel; the host reports it at the next
synchronisation and the context stays usable.

The test makes the waits run out on purpose with the scatter's test hook
(the producer stops feeding its consumers: a flag that nothing sets), checks
the reported status, and then steps on normally.
"""
import time

import numpy as np
import pytest

import simuse_b200 as sg
from simuse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_scatter_wait_limit_reports_an_error_and_the_context_stays_usable():
    spec = W.lif_balanced(n=20_000, k_in=100, seed=3, ext_rate_hz=4000.0, ext_weight=100.0)
    net = sg.Network(0)
    pop = W.build_lif(net, spec)
    net.build()
    assert net.scatter_mode == "exact"
    net.step(50)
    net.synchronize()
    assert net.events_total > 0
    net.debug_stall_scatter(True)
    t0 = time.time()
    net.step(1)
    with pytest.raises(sg.SimuseError, match="timed out"):
        net.synchronize()
    assert time.time() - t0 < 30
    net.synchronize()  # reported once
    net.debug_stall_scatter(False)
    ev = net.events_total
    net.step(20)
    net.synchronize()
    assert net.events_total > ev
    assert np.isfinite(net.state(pop, 0)).all()
    net.close()
