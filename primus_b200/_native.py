"""ctypes binding of libprimus_gpu.so (the C ABI declared in include/primus_gpu.h).

The product path has no CPU fallback: if the library is missing, importing this
module raises, and every call that fails on the device raises PrimusGpuError
with the library's status code and message.
"""
from __future__ import annotations

import ctypes as C
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprimus_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "primus_gpu.h")

u64p = C.POINTER(C.c_uint64)
vp = C.c_void_p

PG_OK = 0
STATUS = {}


class PrimusGpuError(RuntimeError):
    def __init__(self, status: int, where: str, message: str):
        self.status = status
        self.where = where
        self.message = message
        super().__init__(f"{where}: {STATUS.get(status, status)}: {message}")


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m primus_b200.build` (nvcc, sm_100a). "
            "There is no CPU fallback.")
    return C.CDLL(LIB_PATH)


_lib = _load()

# ---- signatures: parsed from the header so that every declared entry point is typed
_CTYPE = {
    "int": C.c_int, "uint32_t": C.c_uint32, "int32_t": C.c_int32, "uint64_t": C.c_uint64, "size_t": C.c_size_t,
    "float": C.c_float, "double": C.c_double, "void": None, "const char *": C.c_char_p, "uint8_t": C.c_uint8,
}


def _parse_header(path: str):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    text = re.sub(r"//[^\n]*", " ", text)
    decls = {}
    for m in re.finditer(r"([A-Za-z_][\w\s\*]*?)\b(pg_\w+)\s*\(([^)]*)\)\s*;", text):
        ret, name, args = m.group(1).strip(), m.group(2), m.group(3).strip()
        decls[name] = (ret, [a.strip() for a in args.split(",")] if args and args != "void" else [])
    return decls


def _ctype_of(decl: str):
    d = " ".join(decl.replace("*", " * ").split())
    base = re.sub(r"\b[a-z_][a-z0-9_]*$", "", d).strip() if not d.endswith("*") else d
    if "*" in base:
        if base.startswith("const char"):
            return C.c_char_p
        return C.c_void_p
    base = base.replace("const ", "").strip()
    return _CTYPE.get(base, C.c_void_p)


DECLS = _parse_header(HEADER)
for _name, (_ret, _args) in DECLS.items():
    _f = getattr(_lib, _name)
    _r = _ret.replace("const ", "const ").strip()
    if _r.endswith("*"):
        _f.restype = C.c_char_p if "char" in _r else C.c_void_p
    else:
        _f.restype = _CTYPE.get(_r, C.c_int)
    _f.argtypes = [_ctype_of(a) for a in _args]

for _code, _nm in enumerate(["PG_OK", "PG_ERR_INVALID_ARGUMENT", "PG_ERR_NO_PRIMITIVE_ROOT", "PG_ERR_DEGREE_TOO_LARGE",
                             "PG_ERR_NOT_COPRIME", "PG_ERR_UNSUPPORTED", "PG_ERR_OUT_OF_MEMORY", "PG_ERR_CUDA",
                             "PG_ERR_TIMEOUT", "PG_ERR_REJECTED"]):
    globals()[_nm] = _code
    STATUS[_code] = _lib.pg_status_string(_code).decode()


def lib():
    return _lib


def check(status: int, where: str):
    if status != PG_OK:
        raise PrimusGpuError(status, where, _lib.pg_last_error().decode())


def call(name: str, *args):
    check(getattr(_lib, name)(*args), name)


def ptr(a: np.ndarray) -> int:
    assert a.flags.c_contiguous
    return a.ctypes.data


# ---------------------------------------------------------------- device objects

class Stream:
    def __init__(self):
        h = vp()
        call("pg_stream_create", C.byref(h))
        self.h = h.value

    def synchronize(self):
        call("pg_stream_synchronize", self.h)

    def close(self):
        if self.h:
            _lib.pg_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _sh(stream):
    return None if stream is None else stream.h


class Event:
    def __init__(self):
        h = vp()
        call("pg_event_create", C.byref(h))
        self.h = h.value

    def record(self, stream=None):
        call("pg_event_record", self.h, _sh(stream))

    def elapsed_ms(self, end: "Event") -> float:
        ms = C.c_float()
        call("pg_event_elapsed_ms", self.h, end.h, C.byref(ms))
        return ms.value

    def __del__(self):
        try:
            if self.h:
                _lib.pg_event_destroy(self.h)
        except Exception:
            pass


class DeviceBuffer:
    """A device array of uint64 (owned; freed on close / garbage collection)."""

    def __init__(self, count: int):
        self.count = int(count)
        h = vp()
        call("pg_malloc", C.byref(h), self.count * 8)
        self.ptr = h.value or 0

    @classmethod
    def from_numpy(cls, a: np.ndarray, stream=None) -> "DeviceBuffer":
        a = np.ascontiguousarray(a, dtype=np.uint64)
        b = cls(a.size)
        b.upload(a, stream)
        return b

    def upload(self, a: np.ndarray, stream=None):
        a = np.ascontiguousarray(a, dtype=np.uint64)
        assert a.size <= self.count
        call("pg_memcpy_h2d", self.ptr, ptr(a), a.size * 8, _sh(stream))
        if stream is None:
            call("pg_stream_synchronize", None)
        else:
            stream.synchronize()

    def numpy(self, shape=None, stream=None) -> np.ndarray:
        out = np.empty(self.count, dtype=np.uint64)
        call("pg_memcpy_d2h", ptr(out), self.ptr, self.count * 8, _sh(stream))
        call("pg_stream_synchronize", _sh(stream))
        return out.reshape(shape) if shape is not None else out

    @classmethod
    def from_bytes(cls, data: bytes) -> "DeviceBuffer":
        """The reference's from_bytes: little-endian u64 words (len(data) must be a multiple of 8)."""
        b = cls(len(data) // 8)
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        call("pg_from_bytes", b.ptr, b.count, buf, len(data))
        return b

    def to_bytes(self) -> bytes:
        """The reference's to_bytes: the words as little-endian bytes."""
        buf = (C.c_uint8 * (self.count * 8))()
        call("pg_to_bytes", self.ptr, self.count, buf, self.count * 8)
        return bytes(buf)

    def zero(self, stream=None):
        call("pg_memset", self.ptr, 0, self.count * 8, _sh(stream))

    def close(self):
        if self.ptr:
            _lib.pg_free(self.ptr)
            self.ptr = 0

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count() -> int:
    c = C.c_int(0)
    st = _lib.pg_device_count(C.byref(c))
    return c.value if st == PG_OK else 0


def synchronize():
    call("pg_device_synchronize")


def launch_count() -> int:
    return int(_lib.pg_launch_count())
