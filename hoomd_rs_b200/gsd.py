"""GSD files through libhmc_b200.so, with hoomd-gsd's API names.

``GsdFile`` mirrors ``hoomd_gsd::file_layer::GsdFile`` (hoomd-gsd/src/file_layer.rs) and
``HoomdGsdFile`` / ``Frame`` mirror ``hoomd_gsd::hoomd`` (hoomd-gsd/src/hoomd.rs), so a frame
is written as::

    f = HoomdGsdFile.create("trajectory.gsd")
    f.append_frame(1000).configuration_box([L, L, L, 0, 0, 0]).particles_position(pos).end()
    f.append_microstate(microstate).log_scalar("acceptance", 0.3).end()   # from device state
    f.close()

All file work is native (``hmc_gsd_*`` in the library); ``append_microstate`` converts the
device-resident state to FP32 on the GPU. Errors raise ``GsdError`` whose ``kind`` names the
reference's error variant (``"NotWritable"``, ``"DuplicateChunkName"``, ``"InvalidColumns"``,
``"InvalidType"``, ``"ChunkNotFound"``, ...).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import OK, HmcError, _vp, hmc_gsd_chunk, hmc_gsd_info, load_library

# hmc_gsd_type (file_layer.rs DataType)
U8, U16, U32, U64, I8, I16, I32, I64, F32, F64, STRING = range(1, 12)
_TYPE_OF = {np.dtype(np.uint8): U8, np.dtype(np.uint16): U16, np.dtype(np.uint32): U32,
            np.dtype(np.uint64): U64, np.dtype(np.int8): I8, np.dtype(np.int16): I16, np.dtype(np.int32): I32,
            np.dtype(np.int64): I64, np.dtype(np.float32): F32, np.dtype(np.float64): F64}
_DTYPE_OF = {v: k for k, v in _TYPE_OF.items()}
_DTYPE_OF[STRING] = np.dtype(np.uint8)

# hmc_gsd_error -> the reference's error variant
KINDS = {0: "Ok", 1: "IO", 2: "NameTooLong", 3: "NotWritable", 4: "DuplicateChunkName", 5: "NameListOverflow",
         6: "InvalidColumns", 7: "InvalidType", 8: "ChunkNotFound", 9: "InconsistentLength",
         10: "InvalidFileIdentifier", 11: "UnsupportedVersion", 12: "IndexOutOfBounds", 13: "NameListOutOfBounds",
         14: "NameListNotTerminated", 15: "CorruptIndexEntry", 16: "InvalidString", 17: "ChunkTooLarge"}


class GsdError(HmcError):
    def __init__(self, status: int, kind: str, message: str):
        super().__init__(status, f"{kind}: {message}")
        self.kind = kind


def _check(status: int):
    if status != OK:
        lib = load_library()
        raise GsdError(status, KINDS.get(lib.hmc_gsd_last_error(), "Unknown"), lib.hmc_last_error_message().decode())


def _path(p) -> bytes:
    return os.fsencode(os.fspath(p))


@dataclass(frozen=True)
class IndexEntry:
    """One index entry (file_layer.rs IndexEntry)."""

    frame: int
    rows: int
    columns: int
    data_type: int
    location: int
    id: int


class Mode:
    READ = 0
    WRITE = 1


class GsdFile:
    """A GSD file (file_layer.rs GsdFile). Close it (or use ``with``) to synchronise."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def create(cls, path, application: str, schema: str, schema_version=(1, 0)):
        h = _vp()
        _check(load_library().hmc_gsd_create(_path(path), application.encode(), schema.encode(),
                                             schema_version[0], schema_version[1], 0, C.byref(h)))
        return cls(h)

    @classmethod
    def create_new(cls, path, application: str, schema: str, schema_version=(1, 0)):
        h = _vp()
        _check(load_library().hmc_gsd_create(_path(path), application.encode(), schema.encode(),
                                             schema_version[0], schema_version[1], 1, C.byref(h)))
        return cls(h)

    @classmethod
    def open(cls, path, mode: int = Mode.READ):
        h = _vp()
        _check(load_library().hmc_gsd_open(_path(path), int(mode), C.byref(h)))
        return cls(h)

    def close(self):
        h, self._h = getattr(self, "_h", None), None
        if h:
            _check(load_library().hmc_gsd_close(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load_library().hmc_gsd_close(h)
            self._h = None

    # ---- writing
    def _write(self, name: str, values: np.ndarray, columns: int, dtype=None):
        a = np.ascontiguousarray(values, dtype=dtype)
        t = _TYPE_OF.get(a.dtype)
        if t is None:
            raise TypeError(f"no GSD type for {a.dtype}")
        rows = a.size // columns if columns else 0
        _check(load_library().hmc_gsd_write_chunk(self._h, name.encode(), t, rows, columns,
                                                  a.ctypes.data if a.size else None))

    def write_scalars(self, name: str, data, dtype=None):
        """write_scalars (file_layer.rs:1735-1749): one column."""
        a = np.ascontiguousarray(data, dtype=dtype).reshape(-1)
        self._write(name, a, 1)

    def write_arrays(self, name: str, data, dtype=None):
        """write_arrays (file_layer.rs:1790-1830): rows of M >= 1 values."""
        a = np.asarray(data, dtype=dtype)
        columns = a.shape[1] if a.ndim == 2 else 0
        if a.ndim != 2:
            a = a.reshape(0, 0) if a.size == 0 else a
        self._write(name, a, columns)

    def write_string(self, name: str, data: str):
        b = data.encode()
        buf = C.create_string_buffer(b, len(b))
        _check(load_library().hmc_gsd_write_chunk(self._h, name.encode(), STRING, len(b), 1, buf))

    def write_strings_array(self, name: str, strings: Sequence[str]):
        arr = (C.c_char_p * len(strings))(*[s.encode() for s in strings])
        _check(load_library().hmc_gsd_write_strings(self._h, name.encode(), arr, len(strings)))

    def end_frame(self):
        _check(load_library().hmc_gsd_end_frame(self._h))

    def sync_all(self):
        _check(load_library().hmc_gsd_sync(self._h))

    # ---- facts
    def _info(self) -> hmc_gsd_info:
        i = hmc_gsd_info()
        _check(load_library().hmc_gsd_get_info(self._h, C.byref(i)))
        return i

    def n_frames(self) -> int:
        return self._info().n_frames

    def application(self) -> str:
        return self._info().application.decode()

    def schema(self) -> str:
        return self._info().schema.decode()

    def schema_version(self):
        i = self._info()
        return (i.schema_major, i.schema_minor)

    def mode(self) -> int:
        return Mode.WRITE if self._info().writable else Mode.READ

    def file_length(self) -> int:
        return self._info().file_length

    def info(self) -> dict:
        i = self._info()
        return {f: getattr(i, f) for f, _ in hmc_gsd_info._fields_}

    @property
    def maximum_write_buffer_size(self) -> int:
        return self._info().maximum_write_buffer_size

    @maximum_write_buffer_size.setter
    def maximum_write_buffer_size(self, n: int):
        _check(load_library().hmc_gsd_set_maximum_write_buffer_size(self._h, int(n)))

    def name_id(self) -> dict:
        lib = load_library()
        out, buf = {}, C.create_string_buffer(1 << 16)
        for i in range(self._info().n_names):
            _check(lib.hmc_gsd_name(self._h, i, buf, len(buf)))
            out[buf.value.decode()] = i
        return out

    # ---- reading
    def find_chunk(self, frame: int, name: str) -> Optional[IndexEntry]:
        c, found = hmc_gsd_chunk(), C.c_int()
        _check(load_library().hmc_gsd_find_chunk(self._h, frame, name.encode(), C.byref(c), C.byref(found)))
        if not found.value:
            return None
        return IndexEntry(c.frame, c.rows, c.columns, c.type, c.location, c.id)

    def _read(self, frame: int, name: str, t: int, columns: int) -> np.ndarray:
        lib = load_library()
        e = self.find_chunk(frame, name)
        rows = C.c_uint64()
        if e is None or e.columns != columns or e.data_type != t:
            # let the library report the reference's error for this read
            _check(lib.hmc_gsd_read_chunk(self._h, frame, name.encode(), t, columns, None, 0, C.byref(rows)))
        out = np.empty((e.rows, columns), dtype=_DTYPE_OF[t])
        _check(lib.hmc_gsd_read_chunk(self._h, frame, name.encode(), t, columns,
                                      out.ctypes.data if out.size else None, out.nbytes, C.byref(rows)))
        return out

    def iter_scalars(self, frame: int, name: str, dtype) -> np.ndarray:
        """iter_scalars (file_layer.rs:1507-1545): a 1-D array of the chunk's values."""
        return self._read(frame, name, _TYPE_OF[np.dtype(dtype)], 1).reshape(-1)

    def iter_arrays(self, frame: int, name: str, dtype, m: int) -> np.ndarray:
        """iter_arrays (file_layer.rs:1577-1617): rows x m."""
        return self._read(frame, name, _TYPE_OF[np.dtype(dtype)], m)

    def read_string(self, frame: int, name: str) -> str:
        return self._read(frame, name, STRING, 1).tobytes().decode()


class HoomdGsdFile(GsdFile):
    """A GSD file with the HOOMD schema, version 1.4 (hoomd.rs HoomdGsdFile)."""

    @classmethod
    def create(cls, path, application: Optional[str] = None):
        h = _vp()
        _check(load_library().hmc_gsd_create_hoomd(_path(path), None if application is None else application.encode(),
                                                   0, C.byref(h)))
        return cls(h)

    @classmethod
    def create_new(cls, path, application: Optional[str] = None):
        h = _vp()
        _check(load_library().hmc_gsd_create_hoomd(_path(path), None if application is None else application.encode(),
                                                   1, C.byref(h)))
        return cls(h)

    @classmethod
    def open(cls, path, mode: int = Mode.WRITE):
        return super().open(path, mode)

    def set_auto_sync_delay(self, seconds: float):
        _check(load_library().hmc_gsd_set_auto_sync_delay(self._h, float(seconds)))

    def append_frame(self, step: int) -> "Frame":
        """append_frame (hoomd.rs:343-350): writes configuration/step."""
        _check(load_library().hmc_gsd_append_frame(self._h, int(step)))
        return Frame(self)

    def append_microstate(self, microstate) -> "Frame":
        """AppendMicrostate::append_microstate (hoomd-microstate/src/append.rs:115-129) from the
        GPU-resident state of a ``Microstate``: step, FP32 site positions and orientations,
        dimensions and box. Add more chunks to the returned frame, then ``end()`` it."""
        _check(load_library().hmc_gsd_append_system(self._h, microstate._h))
        return Frame(self)


class Frame:
    """An open frame of a HoomdGsdFile (hoomd.rs Frame); chain chunk methods, then ``end()``."""

    def __init__(self, file: HoomdGsdFile):
        self._f = file

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.end()

    def _particles(self, name: str, a: np.ndarray, columns: int):
        t = _TYPE_OF[a.dtype]
        rows = a.size // columns
        _check(load_library().hmc_gsd_frame_particles(self._f._h, name.encode(), t, rows, columns,
                                                      a.ctypes.data if a.size else None))
        return self

    def configuration_dimensions(self, dimensions: int):
        self._f.write_scalars("configuration/dimensions", [dimensions], np.uint8)
        return self

    def configuration_box(self, values):
        """Six box values, stored as FP32 (hoomd.rs:385-398)."""
        self._f.write_scalars("configuration/box", np.asarray(values, dtype=np.float64).astype(np.float32))
        return self

    def particles_position(self, positions):
        a = np.ascontiguousarray(np.asarray(positions, dtype=np.float64).reshape(-1, 3).astype(np.float32))
        return self._particles("particles/position", a, 3)

    def particles_orientation(self, orientations):
        a = np.ascontiguousarray(np.asarray(orientations, dtype=np.float64).reshape(-1, 4).astype(np.float32))
        return self._particles("particles/orientation", a, 4)

    def particles_type_id(self, type_id):
        return self._particles("particles/typeid", np.ascontiguousarray(type_id, dtype=np.uint32).reshape(-1), 1)

    def particles_diameter(self, diameter):
        a = np.ascontiguousarray(np.asarray(diameter, dtype=np.float64).astype(np.float32).reshape(-1))
        return self._particles("particles/diameter", a, 1)

    def particles_types(self, types: Sequence[str]):
        self._f.write_strings_array("particles/types", types)
        return self

    def particles_type_shapes(self, type_shapes: Sequence[str]):
        self._f.write_strings_array("particles/type_shapes", type_shapes)
        return self

    def log_scalar(self, name: str, value, dtype=None):
        self._f.write_scalars(f"log/{name}", np.asarray([value], dtype=dtype))
        return self

    def log_scalars(self, name: str, values, dtype=None):
        self._f.write_scalars(f"log/{name}", values, dtype)
        return self

    def log_arrays(self, name: str, values, dtype=None):
        self._f.write_arrays(f"log/{name}", values, dtype)
        return self

    def end(self):
        """Frame::end (hoomd.rs:766-778): end the frame; sync when the auto-sync delay passed."""
        if self._f is not None:
            _check(load_library().hmc_gsd_frame_end(self._f._h))
            self._f = None


__all__ = ["GsdFile", "HoomdGsdFile", "Frame", "GsdError", "IndexEntry", "Mode", "U8", "U16", "U32", "U64", "I8",
           "I16", "I32", "I64", "F32", "F64", "STRING"]
