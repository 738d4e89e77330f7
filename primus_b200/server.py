"""Python view of the continuous-batching request server (pg_server_*)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as nat
from ._native import PrimusGpuError, call

PG_REQ_POLYMUL, PG_REQ_EXT_PRODUCT, PG_REQ_KEY_SWITCH = 1, 2, 3


class Request(C.Structure):
    _fields_ = [("kind", C.c_int), ("key", C.c_uint32), ("d_a", C.c_void_p), ("d_b", C.c_void_p),
                ("log_n", C.c_uint32), ("moduli_count", C.c_uint32), ("d_in", C.c_void_p), ("d_out", C.c_void_p)]


class ServerConfig(C.Structure):
    _fields_ = [("memory_budget_bytes", C.c_size_t), ("slots", C.c_uint32), ("max_batch", C.c_uint32),
                ("max_queue", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("rejected", C.c_uint64),
                ("batches", C.c_uint64), ("mean_batch", C.c_double), ("p50_us", C.c_double),
                ("p99_us", C.c_double), ("max_us", C.c_double), ("enqueue_mean_us", C.c_double),
                ("enqueue_max_us", C.c_double)]


def polymul_request(a, b, log_n, moduli_count):
    return Request(PG_REQ_POLYMUL, 0, a.ptr, b.ptr, log_n, moduli_count, None, None)


def ext_product_request(key_id, d_in, d_out):
    return Request(PG_REQ_EXT_PRODUCT, key_id, None, None, 0, 0, d_in.ptr, d_out.ptr)


def key_switch_request(key_id, d_in, d_out):
    return Request(PG_REQ_KEY_SWITCH, key_id, None, None, 0, 0, d_in.ptr, d_out.ptr)


class Server:
    def __init__(self, memory_budget_bytes=1 << 30, slots=4, max_batch=256, max_queue=0, polymul_tables=()):
        self.polymul_tables = list(polymul_tables)
        cfg = ServerConfig(memory_budget_bytes, slots, max_batch, max_queue)
        arr = (C.c_void_p * max(1, len(self.polymul_tables)))(*[t.h for t in self.polymul_tables])
        h = C.c_void_p()
        call("pg_server_create", C.byref(cfg), arr, len(self.polymul_tables), C.byref(h))
        self.h = h.value
        self._keys = []

    def register_key(self, kind, table, basis, k_in, k_out, d_key):
        kid = C.c_uint32()
        call("pg_server_register_key", self.h, kind, table.h, basis.h, k_in, k_out, d_key.ptr, C.byref(kid))
        self._keys.append((table, basis, d_key))  # keep them alive
        return kid.value

    def register_hybrid_key(self, ks, k_in, k_out, d_key):
        """Key for PG_REQ_KEY_SWITCH requests run by the hybrid key switch `ks`."""
        kid = C.c_uint32()
        call("pg_server_register_hybrid_key", self.h, ks.h, k_in, k_out, d_key.ptr, C.byref(kid))
        self._keys.append((ks, d_key))
        return kid.value

    def submit(self, req: Request) -> int:
        t = C.c_uint64()
        call("pg_server_submit", self.h, C.byref(req), C.byref(t))
        return t.value

    def try_submit(self, req: Request):
        """(status, ticket): status is the library's code (PG_ERR_REJECTED when refused)."""
        t = C.c_uint64()
        st = nat.lib().pg_server_submit(self.h, C.byref(req), C.byref(t))
        return st, t.value

    def wait(self, ticket: int, timeout_us: int = -1) -> float:
        lat = C.c_double()
        call("pg_server_wait", self.h, ticket, timeout_us, C.byref(lat))
        return lat.value

    def drain(self, timeout_us: int = -1):
        call("pg_server_drain", self.h, timeout_us)

    def stats(self, reset=False) -> dict:
        s = ServerStats()
        call("pg_server_stats", self.h, C.byref(s), int(bool(reset)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}

    def replay(self, reqs, arrival_us) -> np.ndarray:
        """Submit `reqs` at the given arrival offsets (microseconds from the
        start) from a native thread and wait for all; returns per-request
        latencies in microseconds (negative for rejected requests)."""
        n = len(reqs)
        arr = (Request * n)(*reqs)
        t = np.ascontiguousarray(arrival_us, dtype=np.float64)
        out = np.zeros(n, dtype=np.float64)
        call("pg_server_replay", self.h, arr, nat.ptr(t), n, nat.ptr(out))
        return out

    def close(self):
        if getattr(self, "h", None):
            nat.lib().pg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["Server", "Request", "polymul_request", "ext_product_request", "key_switch_request", "PG_REQ_POLYMUL",
           "PG_REQ_EXT_PRODUCT", "PG_REQ_KEY_SWITCH", "PrimusGpuError"]
