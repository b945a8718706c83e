""".taas v2 snapshot container (crates/SiMuse/crates/taas-format).

The library's native writer must give the bytes of the oracle's restatement
of the reference writer (same manifest JSON, CRC32, layout), and its reader
must behave as the reference's tests require (lib.rs:85-277): every kind
round-trips, a wrong kind and a flipped payload byte are rejected, a bad
magic is refused, zstd sections round-trip, the inspector lists names, game
and metadata.  No GPU: the container is host code.
"""
import numpy as np
import pytest

import simuse_b200 as sg
import taas_oracle as T
from simuse_b200 import taas

CREATED = "2026-01-01T00:00:00Z"
ALL_KINDS = [
    ("weights", "f32", np.array([1.0, 2.0, 3.0], np.float32)),
    ("ids", "i32", np.array([10, 20], np.int32)),
    ("big", "i64", np.array([1 << 40], np.int64)),
    ("stamps", "u64", np.array([42], np.uint64)),
    ("mask", "u8", np.array([0, 255, 7], np.uint8)),
    ("name", "str", "creature-7"),
    ("genome", "json", '{"mut":0.01,"tags":["a"]}'),
    ("raw", "blob", bytes([9, 8, 7])),
]


def test_native_writer_gives_the_reference_bytes(tmp_path):
    md = {"world": "meadow", "quote\"and\\slash": "tab\there\nnewline\x01ctl", "ünï": "ça"}
    p = tmp_path / "a.taas"
    taas.write(p, ALL_KINDS, metadata=md, game="dioma", created=CREATED)
    assert p.read_bytes() == T.to_bytes(ALL_KINDS, metadata=md, game="dioma", created=CREATED)
    q = tmp_path / "b.taas"     # no game, no metadata, no sections
    taas.write(q, [], created=CREATED)
    assert q.read_bytes() == T.to_bytes([], created=CREATED)


def test_roundtrip_all_kinds(tmp_path):
    """lib.rs:85-117."""
    p = tmp_path / "a.taas"
    taas.write(p, ALL_KINDS, metadata={"world": "meadow"}, game="dioma")
    for name, kind, v in ALL_KINDS:
        got = taas.read(p, name, kind)
        if kind in ("str", "json", "blob"):
            assert got == v
        else:
            assert np.array_equal(got, v)
    taas.validate(p)
    man, _ = T.parse(p.read_bytes())
    assert man["game"] == "dioma" and man["metadata"] == {"world": "meadow"} and len(man["sections"]) == 8


def test_wrong_kind_rejected(tmp_path):
    """lib.rs:119-125."""
    p = tmp_path / "a.taas"
    taas.write(p, [("x", "i32", np.array([1], np.int32))])
    with pytest.raises(sg.SimuseError, match="is not f32, got i32"):
        taas.read(p, "x", "f32")
    with pytest.raises(sg.SimuseError, match="not found"):
        taas.read(p, "nope", "i32")


def test_corruption_detected(tmp_path):
    """lib.rs:127-139: the manifest still reads; the section fails its CRC."""
    p = tmp_path / "a.taas"
    taas.write(p, [("data", "f32", np.ones(64, np.float32))])
    b = bytearray(p.read_bytes())
    b[-1] ^= 0xFF
    p.write_bytes(bytes(b))
    assert "data" in taas.inspect(p)
    with pytest.raises(sg.SimuseError, match="CRC32 mismatch"):
        taas.read(p, "data", "f32")
    with pytest.raises(sg.SimuseError):
        taas.validate(p)


def test_invalid_magic_and_truncation(tmp_path):
    """lib.rs:141-144, reader.rs:69-121."""
    p = tmp_path / "a.taas"
    p.write_bytes(b"NOTTAAS\x00\x00\x00")
    with pytest.raises(sg.SimuseError, match="too short|magic"):
        taas.validate(p)
    p.write_bytes(b"NOTTAAS\x00\x00\x00\x00\x00\x00\x00")
    with pytest.raises(sg.SimuseError, match="magic"):
        taas.validate(p)
    good = T.to_bytes([("x", "f32", np.ones(4, np.float32))])
    p.write_bytes(good[:-3])                      # payload shorter than the manifest says
    with pytest.raises(sg.SimuseError, match="exceeds data"):
        taas.validate(p)
    p.write_bytes(good[:20])                      # header cut
    with pytest.raises(sg.SimuseError, match="truncated"):
        taas.validate(p)


def _zstd_available(tmp_path):
    try:
        taas.write(tmp_path / "z.taas", [("x", "u8", np.zeros(4, np.uint8))], zstd_level=3)
        return True
    except sg.SimuseError:
        return False


def test_zstd_roundtrip(tmp_path):
    """lib.rs:146-171: raw, compressed, raw sections in one file."""
    if not _zstd_available(tmp_path):
        pytest.skip("libzstd.so.1 not present")
    big = np.arange(4096, dtype=np.float32)
    a, b, c = tmp_path / "a.taas", tmp_path / "b.taas", tmp_path / "c.taas"
    taas.write(a, [("raw", "f32", big)])
    taas.write(b, [("compressed", "f32", big)], zstd_level=3)
    man, _ = T.parse(a.read_bytes())
    assert "compression" not in man["sections"][0]
    import json
    import struct
    data = b.read_bytes()
    (hl,) = struct.unpack("<Q", data[5:13])
    sec = json.loads(data[13:13 + hl])["sections"][0]
    assert sec["compression"] == "zstd" and sec["uncompressed_size"] == big.size * 4 and sec["size"] < big.size * 4
    assert np.array_equal(taas.read(b, "compressed", "f32"), big)
    taas.validate(b)
    taas.write(c, [("raw2", "f32", big)])
    assert np.array_equal(taas.read(c, "raw2", "f32"), big)


def test_inspect_output(tmp_path):
    """lib.rs:192-203 and the listing of inspect.rs:5-53."""
    p = tmp_path / "a.taas"
    taas.write(p, [("test", "f32", np.array([1.0, 2.0, 3.0], np.float32))], metadata={"world": "meadow"},
               game="dioma", created=CREATED)
    out = taas.inspect(p)
    assert out.startswith(f".taas archive: {p}\n   Version: 2.0.0\n   Created: {CREATED}\n   Game:    dioma\n")
    assert "test" in out and "dioma" in out and "meadow" in out
    assert "   test                     f32         12 B  crc=" in out
    assert out.rstrip().endswith("Total size: " + f"{p.stat().st_size} B")


def test_reads_files_of_the_reference_layout(tmp_path):
    """A file assembled by the oracle (the reference layout, with the
    connectome sections of src/python/python/taas_format.rs:16-31) reads
    back section by section."""
    rp = np.array([0, 2, 3, 3], np.int32)
    p = tmp_path / "c.taas"
    p.write_bytes(T.to_bytes([("row_ptr", "i32", rp), ("col_indices", "i32", np.array([1, 2, 0], np.int32)),
                              ("values", "f32", np.array([0.5, -1.0, 2.0], np.float32)),
                              ("nt_types", "f32", np.zeros(3, np.float32)),
                              ("groups", "json", '[{"name":"a","indices":[0,1]}]')], game="dioma"))
    taas.validate(p)
    assert np.array_equal(taas.read(p, "row_ptr", "i32"), rp)
    assert taas.read(p, "groups", "json") == '[{"name":"a","indices":[0,1]}]'


def test_large_sections_use_the_threaded_crc(tmp_path):
    """Sections above a few MB are checksummed in chunks on several threads
    and the chunk CRCs combined; the result must be the single-pass CRC32
    (the oracle's zlib.crc32), and a flipped byte must still be caught."""
    big = np.random.default_rng(5).random(12_000_003).astype(np.float32)   # 48 MB, odd length
    secs = [("small", "u8", np.arange(7, dtype=np.uint8)), ("big", "f32", big)]
    p = tmp_path / "big.taas"
    taas.write(p, secs, created=CREATED)
    assert p.read_bytes() == T.to_bytes(secs, created=CREATED)
    assert np.array_equal(taas.read(p, "big", "f32"), big)
    b = bytearray(p.read_bytes())
    b[len(b) // 2] ^= 0x01
    p.write_bytes(bytes(b))
    with pytest.raises(sg.SimuseError, match="CRC32 mismatch"):
        taas.read(p, "big", "f32")


def test_untrusted_manifests_are_refused(tmp_path):
    """A manifest whose count times element size wraps, whose section runs
    past the file, or whose JSON is malformed is refused, not followed."""
    import json
    import struct
    good = T.to_bytes([("x", "f32", np.ones(4, np.float32))], created=CREATED)
    (hl,) = struct.unpack("<Q", good[5:13])
    man = json.loads(good[13:13 + hl])
    payload = good[13 + hl:]

    def write(m, body=payload):
        h = json.dumps(m, separators=(",", ":")).encode()
        p = tmp_path / "m.taas"
        p.write_bytes(b"TAAS2" + struct.pack("<Q", len(h)) + h + body)
        return p

    bad = json.loads(json.dumps(man))
    bad["sections"][0]["count"] = 2 ** 62 + 4          # 4 * count wraps to 16
    with pytest.raises(sg.SimuseError, match="data len"):
        taas.read(write(bad), "x", "f32")
    bad = json.loads(json.dumps(man))
    bad["sections"][0]["offset"] = 2 ** 64 - 8         # offset + size wraps
    with pytest.raises(sg.SimuseError, match="exceeds data"):
        taas.validate(write(bad))
    p = tmp_path / "j.taas"
    for h in (b'{"version":"2.0.0"', b'{"version":2}', b'[1,2]', b'{"version":"2.0.0","created":"x","sections":[{}]}'):
        p.write_bytes(b"TAAS2" + struct.pack("<Q", len(h)) + h)
        with pytest.raises(sg.SimuseError, match="manifest"):
            taas.validate(p)


def test_empty_sections(tmp_path):
    """Zero-length sections (a network without synapses) round-trip and keep
    the reference writer's bytes."""
    secs = [("row_ptr", "i32", np.zeros(1, np.int32)), ("col_indices", "i32", np.zeros(0, np.int32)),
            ("values", "f32", np.zeros(0, np.float32)), ("name", "str", ""), ("raw", "blob", b"")]
    p = tmp_path / "e.taas"
    taas.write(p, secs, created=CREATED)
    assert p.read_bytes() == T.to_bytes(secs, created=CREATED)
    assert taas.read(p, "values", "f32").size == 0
    assert taas.read(p, "name", "str") == "" and taas.read(p, "raw", "blob") == b""
    taas.validate(p)
