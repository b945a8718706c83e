"""``KuramotoBatch`` — many independent all-to-all Kuramoto populations
advanced together on one GPU by RK4 (sg_kuramoto_* in include/simuse_b200.h).

The reference integrates one population at a time with forward Euler and a
dense or CSR coupling sum (crates/SiMuse/crates/pillars/src/kernels/phase/
kuramoto.rs:42-68, sparse.rs:40-140); for all-to-all coupling the mean-field
identity of crates/SiMuse/crates/t3/src/oscillator.rs:15-20,549 gives the same
coupling term from one O(N) reduction, which is what the device computes at
each RK4 stage.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib


def _p(a):
    return None if a is None else a.ctypes.data


class KuramotoBatch:
    """Instances of sizes ``sizes[i]`` (1..65536) with coupling ``coupling[i]``,
    one time step ``dt`` for all."""

    def __init__(self, sizes, coupling, dt: float, device: int = 0):
        sz = np.ascontiguousarray(sizes, np.uint32)
        k = np.ascontiguousarray(coupling, np.float32)
        if sz.shape != k.shape:
            raise ValueError("sizes and coupling differ in length")
        h = C.c_void_p()
        check(lib().sg_kuramoto_create(C.byref(h), device, sz.size, _p(sz), _p(k), float(dt)))
        self._h = h
        self.sizes = sz.astype(np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])
        self.n_instances = int(sz.size)
        t = C.c_uint64()
        check(lib().sg_kuramoto_total(self._h, C.byref(t)))
        self.total = int(t.value)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sg_kuramoto_destroy(h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_state(self, theta, omega):
        th = np.ascontiguousarray(theta, np.float32)
        om = np.ascontiguousarray(omega, np.float32)
        if th.size != self.total or om.size != self.total:
            raise ValueError(f"theta/omega must hold {self.total} values")
        check(lib().sg_kuramoto_set_state(self._h, _p(th), _p(om)))

    def record(self, max_steps: int):
        check(lib().sg_kuramoto_record(self._h, int(max_steps)))
        self._rec_steps = 0 if max_steps else None

    def run(self, n_steps: int):
        check(lib().sg_kuramoto_run(self._h, int(n_steps)))
        if getattr(self, "_rec_steps", None) is not None:
            self._rec_steps += int(n_steps)

    def synchronize(self):
        check(lib().sg_kuramoto_synchronize(self._h))

    def theta(self) -> np.ndarray:
        out = np.empty(self.total, np.float32)
        check(lib().sg_kuramoto_get_theta(self._h, _p(out)))
        return out

    def instance_theta(self, i: int, theta: np.ndarray | None = None) -> np.ndarray:
        th = self.theta() if theta is None else theta
        return th[self.offsets[i]:self.offsets[i + 1]]

    def r(self) -> np.ndarray:
        """Recorded r(t), shape [n_instances, steps recorded]."""
        steps = getattr(self, "_rec_steps", None) or 0
        out = np.empty((self.n_instances, max(steps, 1)), np.float32)
        n = C.c_uint64()
        check(lib().sg_kuramoto_get_r(self._h, _p(out), out.size, C.byref(n)))
        return out[:, : n.value]

    def r_mean(self) -> np.ndarray:
        out = np.empty(self.n_instances, np.float64)
        check(lib().sg_kuramoto_get_r_mean(self._h, _p(out)))
        return out

    def stream(self) -> int:
        s = C.c_void_p()
        check(lib().sg_kuramoto_stream(self._h, C.byref(s)))
        return s.value or 0
