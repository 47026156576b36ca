"""GSD file layer and HOOMD schema frames through the C ABI (hmc_gsd_*), on the host.

The cases restate the reference's own tests of hoomd-gsd (file_layer.rs tests module,
hoomd.rs tests module) and compare the library's files byte for byte with the oracle's
restatement of the writer (oracle/gsd_oracle.py) over random sequences of writes, frames,
syncs and buffer sizes that exercise buffer flushes and the growth of the index and the name
list. No GPU is used: the file layer makes no CUDA call.
"""
from __future__ import annotations

import os
import struct

import numpy as np
import pytest

from hoomd_rs_b200.gsd import GsdError, GsdFile, HoomdGsdFile, Mode
from hoomd_rs_b200 import gsd as G
from oracle import gsd_oracle as O

NP = {G.U8: np.uint8, G.U16: np.uint16, G.U32: np.uint32, G.U64: np.uint64, G.I8: np.int8, G.I16: np.int16,
      G.I32: np.int32, G.I64: np.int64, G.F32: np.float32, G.F64: np.float64}

INITIAL_SIZE = 256 + 32 * 128 + 1024


def kind(excinfo):
    return excinfo.value.kind


# ---- file_layer.rs tests ----------------------------------------------------------------

def test_create_new(tmp_path):
    path = tmp_path / "test.gsd"
    GsdFile.create_new(path, "application", "schema", (12, 42)).close()
    f = GsdFile.open(path, Mode.READ)
    assert f.application() == "application"
    assert f.schema() == "schema"
    assert f.schema_version() == (12, 42)
    assert f.n_frames() == 0
    assert f.name_id() == {}
    f.close()
    with pytest.raises(GsdError) as e:
        GsdFile.create_new(path, "application", "schema", (12, 42))
    assert kind(e) == "IO"


def test_new_file_layout(tmp_path):
    path = tmp_path / "test.gsd"
    GsdFile.create(path, "application", "schema", (12, 42)).close()
    b = path.read_bytes()
    assert len(b) == INITIAL_SIZE
    magic, il, ia, nl, na, sv, gv = struct.unpack_from("=QQQQQII", b, 0)
    assert (magic, il, ia, nl, na) == (0x65DF65DF65DF65DF, 256, 128, 256 + 32 * 128, 16)
    assert (sv, gv) == ((12 << 16) | 42, (2 << 16) | 1)
    assert b[48:60] == b"application\0" and b[112:119] == b"schema\0"
    assert b[256:] == bytes(len(b) - 256)


def test_open_write(tmp_path):
    path = tmp_path / "test.gsd"
    GsdFile.create_new(path, "application", "schema", (12, 42)).close()
    f = GsdFile.open(path, Mode.WRITE)
    f.write_scalars("a", [1], np.int32)
    f.end_frame()
    f.sync_all()
    f.close()
    r = GsdFile.open(path)
    assert list(r.iter_scalars(0, "a", np.int32)) == [1]


def test_create_errors(tmp_path):
    path = tmp_path / "test.gsd"
    GsdFile.create(path, "application", "schema", (12, 42)).close()
    with pytest.raises(GsdError) as e:
        GsdFile.create(path, "a" * 64, "schema", (1, 0))
    assert kind(e) == "NameTooLong"
    with pytest.raises(GsdError) as e:
        GsdFile.create(path, "a", "s" * 64, (1, 0))
    assert kind(e) == "NameTooLong"
    GsdFile.create(path, "a" * 63, "s" * 63, (1, 0)).close()
    r = GsdFile.open(path)
    assert r.application() == "a" * 63 and r.schema() == "s" * 63


def test_maximum_write_buffer_size(tmp_path):
    f = GsdFile.create(tmp_path / "test.gsd", "a", "s", (1, 0))
    f.maximum_write_buffer_size = 8
    assert f.maximum_write_buffer_size == 8
    initial = os.path.getsize(tmp_path / "test.gsd")
    assert initial == f.file_length() == INITIAL_SIZE
    f.write_scalars("a", [1], np.uint64)
    f.end_frame()
    assert os.path.getsize(tmp_path / "test.gsd") == f.file_length() == initial + 8


def test_sync_all(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    initial = os.path.getsize(path)
    f.write_scalars("a", [1], np.uint64)
    f.end_frame()
    assert os.path.getsize(path) == f.file_length() == initial
    f.sync_all()
    assert os.path.getsize(path) == f.file_length() == initial + 8


def test_pending_index(tmp_path):
    f = GsdFile.create(tmp_path / "test.gsd", "a", "s", (1, 0))
    f.write_scalars("a", [1], np.int32)
    f.end_frame()
    for i, name in enumerate("abcdefgh"):
        f.write_scalars(name, [i + 1], np.int32)
    assert f.n_frames() == 0
    f.sync_all()
    assert f.find_chunk(0, "a") is not None
    assert f.n_frames() == 1
    for name in "abcdefgh":
        assert f.find_chunk(1, name) is None
    f.end_frame()
    assert f.n_frames() == 1
    f.sync_all()
    assert f.n_frames() == 2
    for name in "abcdefgh":
        assert f.find_chunk(1, name) is not None


def test_all_types(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    data = {"u8": (np.uint8, [1, 2, 3]), "u16": (np.uint16, [4, 5, 6]), "u32": (np.uint32, [7, 8, 9]),
            "u64": (np.uint64, [10, 11, 12]), "i8": (np.int8, [-1, -2, -3]), "i16": (np.int16, [-4, -5, -6]),
            "i32": (np.int32, [-7, -8, -9]), "i64": (np.int64, [-10, -11, -12]),
            "f32": (np.float32, [13.0, 14.0, 15.0]), "f64": (np.float64, [16.0, 17.0, 18.0])}
    for name, (t, v) in data.items():
        f.write_scalars(name, v, t)
    f.write_string("string", "Test string.")
    f.end_frame()
    f.close()
    r = GsdFile.open(path)
    assert r.n_frames() == 1
    for name, (t, v) in data.items():
        a = r.iter_scalars(0, name, t)
        assert a.dtype == np.dtype(t) and list(a) == v
        assert r.find_chunk(0, name).data_type == G._TYPE_OF[np.dtype(t)]
    assert r.read_string(0, "string") == "Test string."
    assert r.find_chunk(0, "string").data_type == G.STRING


def test_dimensions(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    initial = os.path.getsize(path)
    f.write_scalars("a", [], np.uint64)
    f.end_frame()
    f.write_scalars("b", [1, 2, 3, 4, 5, 6], np.uint64)
    f.write_arrays("c", [[1, 2, 3], [4, 5, 6]], np.uint64)
    f.end_frame()
    f.sync_all()
    assert os.path.getsize(path) == f.file_length() == initial + 12 * 8
    f.close()
    r = GsdFile.open(path)
    assert r.n_frames() == 2
    assert r.iter_scalars(0, "a", np.uint64).size == 0
    assert list(r.iter_scalars(1, "b", np.uint64)) == [1, 2, 3, 4, 5, 6]
    assert r.iter_arrays(1, "b", np.uint64, 1).tolist() == [[1], [2], [3], [4], [5], [6]]
    assert r.iter_arrays(1, "c", np.uint64, 3).tolist() == [[1, 2, 3], [4, 5, 6]]
    ea, eb, ec = r.find_chunk(0, "a"), r.find_chunk(1, "b"), r.find_chunk(1, "c")
    assert (ea.frame, ea.rows, ea.columns, ea.data_type) == (0, 0, 1, G.U64)
    assert (eb.frame, eb.rows, eb.columns, eb.data_type) == (1, 6, 1, G.U64)
    assert (ec.frame, ec.rows, ec.columns, ec.data_type) == (1, 2, 3, G.U64)


def test_invalid_writes(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    with pytest.raises(GsdError) as e:
        f.write_arrays("a", np.zeros((0, 0), dtype=np.uint64))
    assert kind(e) == "InvalidColumns"
    f.close()
    r = GsdFile.open(path, Mode.READ)
    with pytest.raises(GsdError) as e:
        r.write_scalars("a", [], np.uint64)
    assert kind(e) == "NotWritable"
    with pytest.raises(GsdError) as e:
        r.end_frame()
    assert kind(e) == "NotWritable"
    with pytest.raises(GsdError) as e:
        r.sync_all()
    assert kind(e) == "NotWritable"


def test_duplicate_chunk_name(tmp_path):
    f = GsdFile.create(tmp_path / "test.gsd", "a", "s", (1, 0))
    f.write_scalars("a", [1], np.int32)
    with pytest.raises(GsdError) as e:
        f.write_scalars("a", [1, 2], np.int32)
    assert kind(e) == "DuplicateChunkName"


def test_read_invalid_reads(tmp_path):
    f = GsdFile.create(tmp_path / "test.gsd", "a", "s", (1, 0))
    f.write_scalars("a", [1], np.uint64)
    f.write_arrays("b", [[1, 2], [3, 4]], np.uint64)
    f.end_frame()
    f.sync_all()
    cases = [(lambda: f.iter_scalars(0, "a", np.uint32), "InvalidType"),
             (lambda: f.iter_scalars(0, "b", np.uint64), "InvalidColumns"),
             (lambda: f.iter_arrays(0, "a", np.uint64, 2), "InvalidColumns"),
             (lambda: f.iter_arrays(0, "b", np.uint64, 8), "InvalidColumns"),
             (lambda: f.iter_scalars(1, "a", np.uint32), "ChunkNotFound"),
             (lambda: f.iter_scalars(0, "q", np.uint32), "ChunkNotFound")]
    for call, k in cases:
        with pytest.raises(GsdError) as e:
            call()
        assert kind(e) == k


def test_chunk_name_limit(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    for i in range(0xFFFF):
        f.write_scalars(f"{i:x}", [], np.uint64)
    with pytest.raises(GsdError) as e:
        f.write_scalars(f"{0xFFFF:x}", [], np.uint64)
    assert kind(e) == "NameListOverflow"
    f.close()
    r = GsdFile.open(path)
    names = r.name_id()
    assert len(names) == 0xFFFF
    assert all(f"{i:x}" in names for i in range(0xFFFF))
    assert os.path.getsize(path) == r.file_length()


def test_expand_index_multi(tmp_path):
    path = tmp_path / "test.gsd"
    f = GsdFile.create(path, "a", "s", (1, 0))
    for i in range(1024):
        f.write_scalars(f"{i:x}", [i], np.uint16)
    f.end_frame()
    f.sync_all()
    f.close()
    r = GsdFile.open(path)
    assert r.info()["index_entries"] == 1024
    for i in range(1024):
        assert list(r.iter_scalars(0, f"{i:x}", np.uint16)) == [i]


def test_string(tmp_path):
    f = GsdFile.create(tmp_path / "test.gsd", "a", "s", (1, 0))
    f.write_string("a", "this is a string")
    f.end_frame()
    f.write_scalars("b", [0, 159, 146, 150], np.uint8)
    f.end_frame()
    f.sync_all()
    assert f.read_string(0, "a") == "this is a string"
    with pytest.raises(GsdError) as e:
        f.read_string(1, "b")
    assert kind(e) == "InvalidType"


# ---- hoomd.rs tests -----------------------------------------------------------------------

def test_hoomd_create_and_create_new(tmp_path):
    path = tmp_path / "test.gsd"
    HoomdGsdFile.create(path).close()
    r = GsdFile.open(path)
    assert r.application().startswith("hoomd-rs")
    assert r.schema() == "hoomd" and r.schema_version() == (1, 4)
    assert r.n_frames() == 0 and r.name_id() == {}
    r.close()
    with pytest.raises(GsdError) as e:
        HoomdGsdFile.create_new(path)
    assert kind(e) == "IO"
    w = HoomdGsdFile.open(path)
    assert w.mode() == Mode.WRITE
    w.close()


def test_hoomd_frame_chunks(tmp_path):
    path = tmp_path / "test.gsd"
    f = HoomdGsdFile.create(path)
    (f.append_frame(1000).configuration_box([100.0, 50.0, 80.0, 0.0, 0.0, 0.0])
      .particles_position([[0.0, 1.0, 2.0], [3.0, 6.0, 12.0]]).particles_types(["A", "BB"])
      .particles_type_id([0, 1]).particles_diameter([1.0, 2.0]).log_scalar("value", 1.5, np.float64).end())
    f.append_frame(2000).configuration_dimensions(2).end()
    with pytest.raises(GsdError) as e:
        f.append_frame(3000).particles_position([[0.0, 0.0, 0.0]]).particles_type_id([0, 1])
    assert kind(e) == "InconsistentLength"
    f.close()
    r = GsdFile.open(path)
    assert r.n_frames() == 3
    assert list(r.iter_scalars(0, "configuration/step", np.uint64)) == [1000]
    assert list(r.iter_scalars(0, "particles/N", np.uint32)) == [2]
    assert r.iter_arrays(0, "particles/position", np.float32, 3).tolist() == [[0, 1, 2], [3, 6, 12]]
    assert list(r.iter_scalars(0, "configuration/box", np.float32)) == [100, 50, 80, 0, 0, 0]
    types = r.iter_arrays(0, "particles/types", np.int8, 3)
    assert types.tobytes() == b"A\0\0BB\0"
    assert list(r.iter_scalars(0, "particles/typeid", np.uint32)) == [0, 1]
    assert list(r.iter_scalars(0, "particles/diameter", np.float32)) == [1, 2]
    assert list(r.iter_scalars(0, "log/value", np.float64)) == [1.5]
    assert list(r.iter_scalars(1, "configuration/dimensions", np.uint8)) == [2]
    assert r.find_chunk(1, "particles/N") is None
    assert list(r.iter_scalars(2, "particles/N", np.uint32)) == [1]


def test_hoomd_auto_sync(tmp_path):
    path = tmp_path / "test.gsd"
    f = HoomdGsdFile.create(path)
    f.append_frame(1).end()
    assert f.n_frames() == 0  # the default 10 s delay has not passed
    f.set_auto_sync_delay(0.0)
    f.append_frame(2).end()
    assert f.n_frames() == 2
    f.close()


# ---- byte-for-byte against the oracle's writer ------------------------------------------

def _random_ops(rng, n_ops):
    ops, names = [], [f"n{i}/{'x' * int(rng.integers(0, 70))}" for i in range(int(rng.integers(5, 60)))]
    for _ in range(n_ops):
        r = rng.random()
        if r < 0.70:
            t = int(rng.choice(list(NP)))
            rows = int(rng.choice([0, 1, 3, 100, 4000, 70000]))
            cols = int(rng.choice([1, 1, 2, 3, 4]))
            ops.append(("write", str(rng.choice(names)), t, rows, cols))
        elif r < 0.75:
            ops.append(("strings", str(rng.choice(names)), [("s" * int(rng.integers(0, 9))) for _ in range(3)]))
        elif r < 0.80:
            ops.append(("string", str(rng.choice(names)), "txt" * int(rng.integers(0, 5))))
        elif r < 0.93:
            ops.append(("end",))
        elif r < 0.97:
            ops.append(("sync",))
        else:
            ops.append(("buffer", int(rng.choice([0, 8, 1000, 1 << 20]))))
    return ops


def _run(ops, product, oracle, rng):
    for op in ops:
        if op[0] == "write":
            _, name, t, rows, cols = op
            a = (rng.random((rows, cols)) * 100).astype(NP[t])
            p_err = o_err = None
            try:
                if cols == 1:
                    product.write_scalars(name, a.reshape(-1))
                else:
                    product.write_arrays(name, a)
            except GsdError as e:
                p_err = e.kind
            try:
                if cols == 1:
                    oracle.write_scalars(name, a.reshape(-1), t)
                else:
                    oracle.write_arrays(name, a, t)
            except O.OracleError as e:
                o_err = e.kind
            assert p_err == o_err
        elif op[0] == "strings":
            try:
                product.write_strings_array(op[1], op[2])
                oracle.write_strings_array(op[1], op[2])
            except GsdError as e:
                assert e.kind == "DuplicateChunkName"
                with pytest.raises(O.OracleError):
                    oracle.write_strings_array(op[1], op[2])
        elif op[0] == "string":
            try:
                product.write_string(op[1], op[2])
                oracle.write_string(op[1], op[2])
            except GsdError as e:
                assert e.kind == "DuplicateChunkName"
                with pytest.raises(O.OracleError):
                    oracle.write_string(op[1], op[2])
        elif op[0] == "end":
            product.end_frame()
            oracle.end_frame()
        elif op[0] == "sync":
            product.sync_all()
            oracle.sync_all()
        else:
            product.maximum_write_buffer_size = op[1]
            oracle.max_buffer = op[1]


@pytest.mark.parametrize("seed", range(12))
def test_random_writes_byte_identical(tmp_path, seed):
    rng = np.random.default_rng(seed)
    ops = _random_ops(rng, 200)
    path = tmp_path / "p.gsd"
    product = GsdFile.create(path, "app", "schema", (1, 2))
    oracle = O.Writer("app", "schema", (1, 2))
    _run(ops, product, oracle, np.random.default_rng(seed + 1000))
    product.close()
    image = oracle.close()
    assert path.read_bytes() == image
    # each side reads the other's file the same way
    r = O.Reader(path.read_bytes())
    p = GsdFile.open(path)
    assert p.n_frames() == r.n_frames
    for name in r.names:
        for frame in range(r.n_frames):
            e = r.read(frame, name)
            pe = p.find_chunk(frame, name)
            assert (e is None) == (pe is None)
            if e is None:
                continue
            t, n, m, arr = e
            assert (pe.data_type, pe.rows, pe.columns) == (t, n, m)
            if t == G.STRING:
                assert p.read_string(frame, name).encode() == arr.tobytes()
            else:
                got = p.iter_arrays(frame, name, NP[t], m)
                assert got.tobytes() == arr.tobytes()


@pytest.mark.parametrize("seed", range(4))
def test_reopen_and_append_byte_identical(tmp_path, seed):
    rng = np.random.default_rng(100 + seed)
    path = tmp_path / "p.gsd"
    product = GsdFile.create(path, "app", "schema", (3, 1))
    oracle = O.Writer("app", "schema", (3, 1))
    _run(_random_ops(rng, 80) + [("end",)], product, oracle, np.random.default_rng(seed))
    product.close()
    image = oracle.close()
    assert path.read_bytes() == image
    product = GsdFile.open(path, Mode.WRITE)
    oracle = O.Writer(None, None, None, image=image)
    assert product.n_frames() == oracle.file_frame
    _run(_random_ops(rng, 80), product, oracle, np.random.default_rng(seed + 7))
    product.close()
    assert path.read_bytes() == oracle.close()


def test_hoomd_frames_byte_identical(tmp_path):
    rng = np.random.default_rng(5)
    path = tmp_path / "h.gsd"
    product = HoomdGsdFile.create(path, "hoomd-rs-b200")
    oracle = O.Writer("hoomd-rs-b200", "hoomd", (1, 4))
    for frame in range(40):
        n = int(rng.choice([1, 10, 50000]))
        pos = rng.random((n, 3)) * 10
        ori = rng.random((n, 4))
        product.append_frame(frame * 100).particles_position(pos).particles_orientation(ori) \
            .configuration_dimensions(3).configuration_box([10.0, 10.0, 10.0, 0, 0, 0]).end()
        oracle.append_microstate(frame * 100, 3, [10.0, 10.0, 10.0], pos.astype(np.float32), ori.astype(np.float32))
        oracle.end_frame()
        if frame % 7 == 3:
            product.sync_all()
            oracle.sync_all()
    product.close()
    assert path.read_bytes() == oracle.close()


# ---- corrupt files ------------------------------------------------------------------------

def _image():
    w = O.Writer("a", "s", (1, 0))
    w.write_scalars("x", [1, 2, 3], O.U64)
    w.end_frame()
    w.write_scalars("x", [4], O.U64)
    w.end_frame()
    return bytearray(w.close())


@pytest.mark.parametrize("case", ["magic", "version", "index", "namelist", "terminated", "entry_type",
                                  "entry_location", "entry_order", "short"])
def test_corrupt_files(tmp_path, case):
    b = _image()
    expect = {"magic": "InvalidFileIdentifier", "version": "UnsupportedVersion", "index": "IndexOutOfBounds",
              "namelist": "NameListOutOfBounds", "terminated": "NameListNotTerminated",
              "entry_type": "CorruptIndexEntry", "entry_location": "CorruptIndexEntry",
              "entry_order": "CorruptIndexEntry", "short": "IO"}[case]
    if case == "magic":
        b[0] ^= 1
    elif case == "version":
        struct.pack_into("=I", b, 44, 3 << 16)
    elif case == "index":
        struct.pack_into("=Q", b, 16, 1 << 40)
    elif case == "namelist":
        struct.pack_into("=Q", b, 24, len(b))
    elif case == "terminated":
        nl, na = struct.unpack_from("=QQ", b, 24)
        b[nl + na * 64 - 1] = ord("z")
    elif case == "entry_type":
        b[256 + 30] = 12
    elif case == "entry_location":
        struct.pack_into("=Q", b, 256 + 32 + 16, len(b))
    elif case == "entry_order":
        struct.pack_into("=Q", b, 256, 5)  # entry 0 claims frame 5, entry 1 frame 1
    elif case == "short":
        b = b[:100]
    path = tmp_path / "c.gsd"
    path.write_bytes(bytes(b))
    with pytest.raises(GsdError) as e:
        GsdFile.open(path)
    assert kind(e) == expect
    if case != "short":
        with pytest.raises(O.OracleError) as e:
            O.Reader(bytes(b))
        assert e.value.kind == expect


def test_upgrade_minor_version_on_write(tmp_path):
    b = _image()
    struct.pack_into("=I", b, 44, 2 << 16)  # a GSD 2.0 file
    path = tmp_path / "old.gsd"
    path.write_bytes(bytes(b))
    GsdFile.open(path, Mode.READ).close()
    assert struct.unpack_from("=I", path.read_bytes(), 44)[0] == 2 << 16
    GsdFile.open(path, Mode.WRITE).close()
    assert struct.unpack_from("=I", path.read_bytes(), 44)[0] == (2 << 16) | 1


def test_large_chunks_byte_identical(tmp_path):
    # chunks of 40 MB and 24 MB go to the file in parallel pieces; the bytes match one write
    rng = np.random.default_rng(11)
    path = tmp_path / "big.gsd"
    product = GsdFile.create(path, "app", "schema", (1, 0))
    oracle = O.Writer("app", "schema", (1, 0))
    for frame in range(3):
        a = rng.random((5_000_000, 1))
        b = rng.integers(0, 1 << 30, size=(2_000_000, 3)).astype(np.uint32)
        product.write_scalars("a", a.reshape(-1))
        oracle.write_scalars("a", a.reshape(-1), O.F64)
        product.write_string("note", f"frame {frame}")
        oracle.write_string("note", f"frame {frame}")
        product.write_arrays("b", b)
        oracle.write_arrays("b", b, O.U32)
        product.end_frame()
        oracle.end_frame()
    product.close()
    assert path.read_bytes() == oracle.close()
