""".taas v2 snapshot files through the library's native container.

The reference's format (crates/SiMuse/crates/taas-format): named, typed
sections with a CRC32 each and optional zstd, behind a JSON manifest
(TaasWriter / TaasReader / inspect_taas).  These functions need no GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import check, lib

_NP = {"f32": np.float32, "i32": np.int32, "i64": np.int64, "u64": np.uint64, "u8": np.uint8}


def _payload(kind, value):
    """(count, object holding the bytes, its address, byte length) without copying numeric arrays."""
    if kind in _NP:
        a = np.ascontiguousarray(value, dtype=_NP[kind])
        return a.size, a, a.ctypes.data, a.nbytes
    if kind in ("str", "json", "blob"):
        b = value.encode() if isinstance(value, str) else bytes(value)
        return len(b), b, C.cast(C.c_char_p(b), C.c_void_p).value, len(b)
    raise ValueError(f"unknown section kind {kind!r}")


def write(path, sections, metadata=None, game=None, created=None, zstd_level=0):
    """sections: [(name, kind, value)], value an array (numeric kinds), str
    (str/json) or bytes (blob)."""
    n = len(sections)
    enc = [(nm.encode(), kd.encode()) + _payload(kd, v) for nm, kd, v in sections]
    names = (C.c_char_p * max(n, 1))(*[e[0] for e in enc])
    kinds = (C.c_char_p * max(n, 1))(*[e[1] for e in enc])
    counts = (C.c_uint64 * max(n, 1))(*[e[2] for e in enc])
    data = (C.c_void_p * max(n, 1))(*[e[4] for e in enc])
    sizes = (C.c_uint64 * max(n, 1))(*[e[5] for e in enc])
    md = sorted((metadata or {}).items())
    keys = (C.c_char_p * max(len(md), 1))(*[k.encode() for k, _ in md])
    vals = (C.c_char_p * max(len(md), 1))(*[v.encode() for _, v in md])
    check(lib().sg_taas_write(str(path).encode(), created.encode() if created is not None else None,
                              game.encode() if game is not None else None, n, names, kinds, counts, data, sizes,
                              len(md), keys, vals, int(zstd_level)))
    del enc  # the section buffers were borrowed until here


def read(path, name, kind):
    """A section's values: numpy array (numeric kinds), str (str/json) or bytes."""
    size = C.c_uint64()
    check(lib().sg_taas_read(str(path).encode(), name.encode(), kind.encode(), None, 0, C.byref(size)))
    buf = np.empty(max(size.value, 1), np.uint8)
    check(lib().sg_taas_read(str(path).encode(), name.encode(), kind.encode(), buf.ctypes.data, size.value,
                             C.byref(size)))
    raw = buf[:size.value]
    if kind in _NP:
        return raw.view(_NP[kind])
    if kind in ("str", "json"):
        return raw.tobytes().decode()
    return raw.tobytes()


def validate(path):
    check(lib().sg_taas_validate(str(path).encode()))


def inspect(path) -> str:
    need = C.c_uint64()
    check(lib().sg_taas_inspect(str(path).encode(), None, 0, C.byref(need)))
    buf = C.create_string_buffer(need.value)
    check(lib().sg_taas_inspect(str(path).encode(), buf, need.value, C.byref(need)))
    return buf.value.decode()
