""".taas v2 container restated in Python — test infrastructure (the oracle).

Only tests/ load this file.  It restates the reference's format from
crates/SiMuse/crates/taas-format/src:
  lib.rs:54-64        assemble_bytes: b"TAAS2" | u64 LE header length | JSON | payload
  types.rs:74-100     SectionEntry / TaasManifest fields, in declaration order;
                      None options skipped; metadata a BTreeMap (sorted keys)
  writer.rs:75-101    push: CRC32 (crc32fast, IEEE) of the uncompressed bytes,
                      offset = payload length so far, size = stored bytes
  reader.rs:69-158    header parse, offset validation, CRC check after decompression
serde_json writes compact JSON with the same string escapes as Python's
json module with separators (",", ":") and ensure_ascii=False.
Compressed sections are not restated (zstd bytes depend on the library
version); the writer here stores sections uncompressed.
"""
import json
import struct
import zlib

import numpy as np

NP = {"f32": "<f4", "i32": "<i4", "i64": "<i8", "u64": "<u8", "u8": "u1"}


def _payload(kind, value):
    if kind in NP:
        a = np.ascontiguousarray(value, dtype=NP[kind])
        return a.size, a.tobytes()
    b = value.encode() if isinstance(value, str) else bytes(value)
    return len(b), b


def to_bytes(sections, metadata=None, game=None, created="2026-01-01T00:00:00Z"):
    entries, payload = [], b""
    for name, kind, value in sections:
        count, raw = _payload(kind, value)
        entries.append({"name": name, "kind": kind, "count": count, "offset": len(payload), "size": len(raw),
                        "crc32": zlib.crc32(raw) & 0xFFFFFFFF})
        payload += raw
    man = {"version": "2.0.0", "created": created}
    if game is not None:
        man["game"] = game
    man["sections"] = entries
    man["metadata"] = dict(sorted((metadata or {}).items()))
    header = json.dumps(man, separators=(",", ":"), ensure_ascii=False).encode()
    return b"TAAS2" + struct.pack("<Q", len(header)) + header + payload


def parse(data):
    """(manifest dict, {name: uncompressed bytes}) with CRC and bounds checks."""
    if len(data) < 13:
        raise ValueError("File too short")
    if data[:5] != b"TAAS2":
        raise ValueError("Invalid magic")
    (hl,) = struct.unpack("<Q", data[5:13])
    if 13 + hl > len(data):
        raise ValueError("Header truncated")
    man = json.loads(data[13:13 + hl].decode())
    body = data[13 + hl:]
    out = {}
    for s in man["sections"]:
        if s["offset"] + s["size"] > len(body):
            raise ValueError(f"Section '{s['name']}' exceeds data")
        raw = body[s["offset"]:s["offset"] + s["size"]]
        if s.get("compression"):
            raise ValueError("compressed sections are not restated here")
        if "crc32" in s and zlib.crc32(raw) & 0xFFFFFFFF != s["crc32"]:
            raise ValueError(f"Section '{s['name']}' CRC32 mismatch")
        out[s["name"]] = raw
    return man, out


def array(man, secs, name, kind):
    s = next(x for x in man["sections"] if x["name"] == name)
    if s["kind"] != kind:
        raise ValueError(f"Section '{name}' is not {kind}, got {s['kind']}")
    return np.frombuffer(secs[name], dtype=NP[kind])
