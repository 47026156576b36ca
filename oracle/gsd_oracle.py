"""CPU restatement of the GSD file layer of hoomd-gsd (test infrastructure only).

Only ``tests/`` and ``bench.py``'s CPU leg use this module: it is the checker of the
library's hmc_gsd_* entry points, never the product. It restates, in plain Python over an
in-memory file image, what ``GsdFile`` (hoomd-gsd/src/file_layer.rs) does to the bytes of a
file, and parses files the way ``GsdFile::open`` does:

* ``initialize_file`` (file_layer.rs:1077-1116): 256-byte header, 128 zeroed index entries,
  a 1024-byte zeroed name list;
* ``write_details`` (:1936-2015): the chunk's bytes go to the write buffer, which is flushed
  to the end of the file once it holds >= the maximum write buffer size (1 MiB default);
* ``end_frame`` (:2043-2052), ``sync_all`` (:2269-2329), ``flush_names`` (:2229-2260),
  ``expand_name_list_to`` / ``expand_index_to`` (:2331-2436);
* ``from_file`` / ``count_index_entries`` / ``find_chunk`` (:1118-1206, :1362-1470).

The HOOMD schema helpers follow hoomd-gsd/src/hoomd.rs (``append_frame`` :343-350,
``validate_particles_chunk`` :413-437) and hoomd-microstate/src/append.rs:115-129.
"""
from __future__ import annotations

import struct

import numpy as np

NAME_SIZE = 64
ENTRY_SIZE = 32
HEADER_SIZE = 256
MAGIC = 0x65DF65DF65DF65DF
GSD_VERSION = (2, 1)
INITIAL_INDEX_SIZE = 128
INITIAL_NAME_LIST_SIZE = 1024
INITIAL_MAXIMUM_WRITE_BUFFER_SIZE = 1024 * 1024

U8, U16, U32, U64, I8, I16, I32, I64, F32, F64, STRING = range(1, 12)
TYPE_SIZE = {U8: 1, U16: 2, U32: 4, U64: 8, I8: 1, I16: 2, I32: 4, I64: 8, F32: 4, F64: 8, STRING: 1}
NUMPY = {U8: np.uint8, U16: np.uint16, U32: np.uint32, U64: np.uint64, I8: np.int8, I16: np.int16,
         I32: np.int32, I64: np.int64, F32: np.float32, F64: np.float64, STRING: np.uint8}

_ENTRY = struct.Struct("=QQQIHBB")


class OracleError(Exception):
    def __init__(self, kind, msg=""):
        super().__init__(f"{kind}: {msg}")
        self.kind = kind


def encode_header(h) -> bytes:
    b = bytearray(HEADER_SIZE)
    struct.pack_into("=QQQQQ", b, 0, MAGIC, h["index_location"], h["index_allocated"], h["namelist_location"],
                     h["namelist_allocated"])
    struct.pack_into("=II", b, 40, (h["schema_version"][0] << 16) | h["schema_version"][1],
                     (h["gsd_version"][0] << 16) | h["gsd_version"][1])
    app, sch = h["application"].encode(), h["schema"].encode()
    b[48:48 + len(app)] = app
    b[112:112 + len(sch)] = sch
    return bytes(b)


class Writer:
    """GsdFile in write mode over an in-memory image (``self.image``)."""

    def __init__(self, application, schema, schema_version, image=None):
        if image is None:
            if len(application.encode()) > NAME_SIZE - 1 or len(schema.encode()) > NAME_SIZE - 1:
                raise OracleError("NameTooLong")
            self.h = {"index_location": HEADER_SIZE, "index_allocated": INITIAL_INDEX_SIZE,
                      "namelist_location": HEADER_SIZE + ENTRY_SIZE * INITIAL_INDEX_SIZE,
                      "namelist_allocated": INITIAL_NAME_LIST_SIZE // NAME_SIZE,
                      "schema_version": tuple(schema_version), "gsd_version": GSD_VERSION,
                      "application": application, "schema": schema}
            self.image = bytearray(encode_header(self.h))
            self.image += bytes(ENTRY_SIZE * INITIAL_INDEX_SIZE + INITIAL_NAME_LIST_SIZE)
            self.names = {}
            self.name_insert = 0
            self.n_entries = 0
            self.file_frame = 0
        else:
            r = Reader(bytes(image))
            self.image = bytearray(image)
            self.h = r.h
            if self.h["gsd_version"] < GSD_VERSION:
                self.h["gsd_version"] = GSD_VERSION
                self.image[0:HEADER_SIZE] = encode_header(self.h)
            self.names = dict(r.names)
            self.name_insert = r.name_insert
            self.n_entries = len(r.entries)
            self.file_frame = r.n_frames
        self.name_buffer = bytearray()
        self.buffered = []   # entries not in the file: completed frames, then the open frame
        self.pending = 0
        self.frame_names = set()
        self.data = bytearray()
        self.buffer_frame = self.file_frame
        self.max_buffer = INITIAL_MAXIMUM_WRITE_BUFFER_SIZE
        self.particles_n = None

    # -- file primitives
    def _write_at(self, offset, b):
        end = offset + len(b)
        if end > len(self.image):
            self.image += bytes(end - len(self.image))
        self.image[offset:end] = b

    def _flush_data(self):
        if not self.data:
            return False
        self.image += self.data
        self.data = bytearray()
        return True

    def _relocate(self, loc_key, alloc_key, unit, used, needed):
        size = self.h[alloc_key] * unit
        while size <= needed:
            size *= 2
        alloc = -(-size // unit)
        size = alloc * unit
        at = len(self.image)
        old = bytes(self.image[self.h[loc_key]:self.h[loc_key] + used])
        self.image += old
        self.image += bytes(at + size - len(self.image))
        self.h[loc_key] = at
        self.h[alloc_key] = alloc
        self.image[0:HEADER_SIZE] = encode_header(self.h)

    # -- GsdFile
    def get_id(self, name):
        if name in self.names:
            return self.names[name]
        if len(self.names) >= 0xFFFF:
            raise OracleError("NameListOverflow")
        i = len(self.names)
        self.names[name] = i
        self.name_buffer += name.encode() + b"\0"
        return i

    def write(self, name, dtype, rows, columns, payload: bytes):
        location = len(self.image) + len(self.data)
        i = self.get_id(name)
        if i in self.frame_names:
            raise OracleError("DuplicateChunkName")
        self.frame_names.add(i)
        self.data += payload
        self.buffered.append((self.buffer_frame, rows, location, columns, i, dtype, 0))
        self.pending += 1
        if len(self.data) >= self.max_buffer:
            self._flush_data()

    def write_scalars(self, name, values, dtype):
        a = np.ascontiguousarray(values, dtype=NUMPY[dtype]).reshape(-1)
        self.write(name, dtype, a.size, 1, a.tobytes())

    def write_arrays(self, name, values, dtype):
        a = np.ascontiguousarray(values, dtype=NUMPY[dtype])
        if a.ndim != 2 or a.shape[1] == 0:
            raise OracleError("InvalidColumns")
        self.write(name, dtype, a.shape[0], a.shape[1], a.tobytes())

    def write_string(self, name, s):
        b = s.encode()
        self.write(name, STRING, len(b), 1, b)

    def write_strings_array(self, name, strings):
        enc = [s.encode() for s in strings]
        cols = max((len(e) for e in enc), default=0) + 1
        self.write(name, I8, len(enc), cols, b"".join(e + bytes(cols - len(e)) for e in enc))

    def end_frame(self):
        self.buffer_frame += 1
        self.pending = 0
        self.frame_names = set()

    def sync_all(self):
        self._flush_data()
        if self.name_buffer:
            need = self.name_insert + len(self.name_buffer)
            if need > self.h["namelist_allocated"] * NAME_SIZE:
                self._relocate("namelist_location", "namelist_allocated", NAME_SIZE, self.name_insert, need)
            self._write_at(self.h["namelist_location"] + self.name_insert, self.name_buffer)
            self.name_insert += len(self.name_buffer)
            self.name_buffer = bytearray()
        k = len(self.buffered) - self.pending
        if k > 0:
            n = self.n_entries
            if n + k > self.h["index_allocated"]:
                self._relocate("index_location", "index_allocated", ENTRY_SIZE, n * ENTRY_SIZE, (n + k) * ENTRY_SIZE)
            done = sorted(self.buffered[:k], key=lambda e: (e[0], e[4]))
            self._write_at(self.h["index_location"] + n * ENTRY_SIZE, b"".join(_ENTRY.pack(*e) for e in done))
            self.buffered = self.buffered[k:]
            self.n_entries += k
        self.file_frame = self.buffer_frame

    def close(self) -> bytes:
        self.sync_all()
        return bytes(self.image)

    # -- HOOMD schema (hoomd.rs)
    def append_frame(self, step):
        self.write_scalars("configuration/step", [step], U64)
        self.particles_n = None

    def particles(self, name, values, dtype):
        a = np.ascontiguousarray(values, dtype=NUMPY[dtype])
        rows = a.shape[0]
        if self.particles_n is None:
            self.write_scalars("particles/N", [rows], U32)
            self.particles_n = rows
        elif rows != self.particles_n:
            raise OracleError("InconsistentLength")
        if a.ndim == 1:
            self.write_scalars(name, a, dtype)
        else:
            self.write_arrays(name, a, dtype)

    def append_microstate(self, step, dim, edge_lengths, positions_f32, orientations_f32=None):
        """AppendMicrostate::append_microstate (append.rs:115-129); the frame stays open."""
        self.append_frame(step)
        self.particles("particles/position", positions_f32, F32)
        if orientations_f32 is not None:
            self.particles("particles/orientation", orientations_f32, F32)
        self.write_scalars("configuration/dimensions", [dim], U8)
        L = list(edge_lengths) + [0.0] * (3 - len(edge_lengths))
        self.write_scalars("configuration/box", [L[0], L[1], L[2] if dim == 3 else 0.0, 0.0, 0.0, 0.0], F32)


class Reader:
    """GsdFile::open in read mode over the bytes of a file."""

    def __init__(self, image: bytes):
        if len(image) < HEADER_SIZE:
            raise OracleError("IO", "short file")
        magic, il, ia, nl, na = struct.unpack_from("=QQQQQ", image, 0)
        if magic != MAGIC:
            raise OracleError("InvalidFileIdentifier")
        sv, gv = struct.unpack_from("=II", image, 40)

        def cstr(b):
            i = b.find(b"\0")
            return (b if i < 0 else b[:i]).decode()

        self.h = {"index_location": il, "index_allocated": ia, "namelist_location": nl, "namelist_allocated": na,
                  "schema_version": (sv >> 16, sv & 0xFFFF), "gsd_version": (gv >> 16, gv & 0xFFFF),
                  "application": cstr(image[48:HEADER_SIZE]), "schema": cstr(image[112:178])}
        if self.h["gsd_version"][0] != 2:
            raise OracleError("UnsupportedVersion")
        L = len(image)
        if ia == 0 or il + ia * ENTRY_SIZE > L:
            raise OracleError("IndexOutOfBounds")
        if na == 0 or nl + na * NAME_SIZE > L:
            raise OracleError("NameListOutOfBounds")
        namelist = image[nl:nl + na * NAME_SIZE]
        if namelist[-1] != 0:
            raise OracleError("NameListNotTerminated")
        self.names, self.name_insert, pos = {}, 0, 0
        while pos < len(namelist) and namelist[pos] != 0:
            end = namelist.index(b"\0", pos)
            name = namelist[pos:end].decode()
            if name in self.names:
                raise OracleError("DuplicateChunkName")
            self.names[name] = len(self.names)
            self.name_insert += end - pos + 1
            pos = end + 1
        self.image = image
        count = 0
        first = self._entry(0)
        if first[2] != 0 and not self._valid(first):
            raise OracleError("CorruptIndexEntry")
        if first[2] != 0:
            lo, hi = 0, ia
            while True:
                m = (lo + hi) // 2
                em, el = self._entry(m), self._entry(lo)
                if em[2] != 0:
                    if not self._valid(em) or em[0] < el[0]:
                        raise OracleError("CorruptIndexEntry")
                    lo = m
                else:
                    hi = m
                if hi - lo == 1:
                    break
            count = hi
        self.entries = [self._entry(i) for i in range(count)]
        self.n_frames = self.entries[-1][0] + 1 if self.entries else 0

    def _entry(self, i):
        return _ENTRY.unpack_from(self.image, self.h["index_location"] + i * ENTRY_SIZE)

    def _valid(self, e):
        frame, n, loc, m, i, t, flags = e
        return (t in TYPE_SIZE and loc + n * m * TYPE_SIZE[t] <= len(self.image)
                and frame < self.h["index_allocated"] and i < len(self.names) and flags == 0)

    def find_chunk(self, frame, name):
        if frame >= self.n_frames or name not in self.names:
            return None
        i = self.names[name]
        for e in self.entries:
            if e[0] == frame and e[4] == i:
                return e
        return None

    def read(self, frame, name):
        """(type, rows, columns, numpy array of rows x columns) or None."""
        e = self.find_chunk(frame, name)
        if e is None:
            return None
        frame_, n, loc, m, i, t, _ = e
        a = np.frombuffer(self.image, dtype=NUMPY[t], count=n * m, offset=loc).reshape(n, m)
        return t, n, m, a
