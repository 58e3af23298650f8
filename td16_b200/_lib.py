"""ctypes binding of libtd16b200.so (include/td16_b200.h).

The library is the product: importing this module without the built library
raises, and nothing here falls back to a CPU implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libtd16b200.so")

# status codes
OK, NOT_FOUND, OVERFLOW, CUDA_ERROR, INVALID_ARG, TIMEOUT = 0, 1, 2, 3, 4, 5
FLAG_ORDERED, FLAG_PLAIN, FLAG_VERIFY = 1, 2, 4
MAX_N, MAX_DEPTH = 17, 9

INSTANCE_DTYPE = np.dtype([("perm", "<u8"), ("min_rate", "<f4"), ("n_symbols", "u1"),
                           ("offset", "u1"), ("max_moves", "u1"), ("packed", "u1")])
RESULT_DTYPE = np.dtype([("status", "<i4"), ("depth", "<i4"), ("moves", "<u2", (9,)),
                         ("reserved", "<u2"), ("expansions", "<u4")])
assert INSTANCE_DTYPE.itemsize == 16 and RESULT_DTYPE.itemsize == 32


class BatchStats(C.Structure):
    _fields_ = [("expansions", C.c_uint64), ("found", C.c_uint64), ("not_found", C.c_uint64),
                ("errors", C.c_uint64), ("kernel_ms", C.c_float), ("launches", C.c_uint32),
                ("donations", C.c_uint64), ("donated_items", C.c_uint64)]


class TdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None

EXPORTS = ["td_init_slots", "td_search", "td_search_ordered", "td_slot_count", "td_slot_device",
           "td_slot_stream", "td_destroy", "td_prepare_pairs", "td_prepare_perms", "td_synth_perms",
           "td_search_batch", "td_search_batch_device", "td_validate_batch_device",
           "td_positions_to_symbols", "td_configure", "td_configure_steal", "td_int_issue_peak"]


def lib():
    """Loads the engine library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m td16_b200.build` "
                          "(the engine has no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, sz, cp = C.c_void_p, C.c_size_t, C.c_char_p
    L.td_init_slots.argtypes = [C.c_int, C.POINTER(C.c_int), C.c_int, C.c_uint64, cp, sz]
    for name in ("td_search", "td_search_ordered"):
        f = getattr(L, name)
        f.argtypes = [C.c_int, vp, vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                      C.POINTER(C.c_int16), C.POINTER(C.c_int), cp, sz]
    L.td_slot_device.argtypes = [C.c_int]
    L.td_slot_stream.argtypes = [C.c_int]
    L.td_slot_stream.restype = vp
    L.td_prepare_pairs.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, C.POINTER(C.c_int)]
    L.td_prepare_perms.argtypes = [C.c_int, vp, vp, vp, C.c_float, C.c_int, vp, C.POINTER(C.c_int)]
    L.td_synth_perms.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, vp, vp]
    L.td_search_batch.argtypes = [C.c_int, C.c_int, vp, vp, C.c_uint, C.c_uint64,
                                  C.POINTER(BatchStats), cp, sz]
    L.td_search_batch_device.argtypes = [C.c_int, C.c_int, vp, vp, C.c_uint, C.c_uint64, vp, cp, sz]
    L.td_validate_batch_device.argtypes = [C.c_int, vp, vp, vp, vp, cp, sz]
    L.td_positions_to_symbols.argtypes = [vp, C.c_int, vp, C.c_int, vp]
    L.td_positions_to_symbols.restype = None
    L.td_configure.argtypes = [C.c_int, C.c_int]
    L.td_configure_steal.argtypes = [C.c_int, C.c_int, C.c_int]
    _lib = L
    return L


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def check(rc: int, err) -> int:
    if rc in (OK, NOT_FOUND):
        return rc
    raise TdError(rc, err.value.decode(errors="replace") if err is not None else f"status {rc}")


def init_slots(total_slots: int, devices, budget_bytes: int) -> None:
    devs = (C.c_int * max(1, len(devices)))(*devices)
    err = C.create_string_buffer(512)
    check(lib().td_init_slots(int(total_slots), devs, len(devices), int(budget_bytes), err, 512), err)


def destroy() -> None:
    lib().td_destroy()


def search(slot: int, beta, omega, initial_even_cycles: int, min_rate: float, max_moves: int,
           full_sorting: bool = True, ordered: bool = False):
    """One blocking search.  Returns the list of position triples (empty when
    no witness exists)."""
    n = len(beta)
    if len(omega) != n:
        raise TdError(INVALID_ARG, "beta and omega must have equal lengths")
    b = np.zeros(max(1, n), np.uint8)
    o = np.zeros(max(1, n), np.uint8)
    b[:n] = np.frombuffer(bytes(beta), np.uint8)
    o[:n] = np.frombuffer(bytes(omega), np.uint8)
    out = (C.c_int16 * (3 * MAX_DEPTH))()
    depth = C.c_int(0)
    err = C.create_string_buffer(512)
    f = lib().td_search_ordered if ordered else lib().td_search
    rc = f(int(slot), _ptr(b), _ptr(o), n,
           int(initial_even_cycles), float(min_rate), int(max_moves), int(bool(full_sorting)),
           out, C.byref(depth), err, 512)
    check(rc, err)
    return [(out[3 * d], out[3 * d + 1], out[3 * d + 2]) for d in range(depth.value)]


def prepare_pairs(beta: np.ndarray, omega: np.ndarray, n, init, min_rate, max_moves, full) -> np.ndarray:
    count = beta.shape[0]
    beta = np.ascontiguousarray(beta, np.uint8)
    omega = np.ascontiguousarray(omega, np.uint8)
    arrs = [np.ascontiguousarray(np.broadcast_to(v, (count,)), dt) for v, dt in
            ((n, np.uint8), (init, np.int32), (min_rate, np.float32), (max_moves, np.int32), (full, np.uint8))]
    out = np.zeros(count, INSTANCE_DTYPE)
    bad = C.c_int(-1)
    rc = lib().td_prepare_pairs(count, _ptr(beta), _ptr(omega), *[_ptr(a) for a in arrs], _ptr(out), C.byref(bad))
    if rc != OK:
        raise TdError(rc, f"instance {bad.value} is not a valid (beta, omega) pair")
    return out


def prepare_perms(perms: np.ndarray, n, max_moves, min_rate: float = 0.0, full: bool = True) -> np.ndarray:
    count = perms.shape[0]
    perms = np.ascontiguousarray(perms, np.int8)
    assert perms.shape[1] == 16
    n = np.ascontiguousarray(np.broadcast_to(n, (count,)), np.uint8)
    mm = np.ascontiguousarray(np.broadcast_to(max_moves, (count,)), np.int32)
    out = np.zeros(count, INSTANCE_DTYPE)
    bad = C.c_int(-1)
    rc = lib().td_prepare_perms(count, _ptr(perms), _ptr(n), _ptr(mm), float(min_rate), int(full),
                                _ptr(out), C.byref(bad))
    if rc != OK:
        raise TdError(rc, f"permutation {bad.value} is invalid")
    return out


def synth_perms(seed: int, count: int, n_min: int, n_max: int, hard_pct: int, hard_min: int, hard_max: int):
    perms = np.zeros((count, 16), np.int8)
    n = np.zeros(count, np.uint8)
    rc = lib().td_synth_perms(C.c_uint64(seed), count, n_min, n_max, hard_pct, hard_min, hard_max,
                              _ptr(perms), _ptr(n))
    if rc != OK:
        raise TdError(rc, "invalid synthetic-instance parameters")
    return perms, n


def search_batch(slot: int, instances: np.ndarray, flags: int = 0, max_expansions: int = 0):
    """Host arrays in and out.  Returns (results, BatchStats)."""
    instances = np.ascontiguousarray(instances, INSTANCE_DTYPE)
    results = np.zeros(len(instances), RESULT_DTYPE)
    st = BatchStats()
    err = C.create_string_buffer(512)
    rc = lib().td_search_batch(int(slot), len(instances), _ptr(instances), _ptr(results), int(flags),
                               C.c_uint64(max_expansions), C.byref(st), err, 512)
    check(rc, err)
    return results, st


def search_batch_device(slot: int, count: int, d_instances: int, d_results: int, flags: int = 0,
                        max_expansions: int = 0, stream: int | None = None) -> None:
    """Device pointers (ints); enqueues on `stream` (or the slot's)."""
    err = C.create_string_buffer(512)
    rc = lib().td_search_batch_device(int(slot), int(count), C.c_void_p(d_instances), C.c_void_p(d_results),
                                      int(flags), C.c_uint64(max_expansions),
                                      C.c_void_p(stream) if stream else None, err, 512)
    check(rc, err)


def validate_batch_device(count: int, d_instances: int, d_results: int, d_ok: int, stream: int | None = None):
    err = C.create_string_buffer(512)
    rc = lib().td_validate_batch_device(int(count), C.c_void_p(d_instances), C.c_void_p(d_results),
                                        C.c_void_p(d_ok), C.c_void_p(stream) if stream else None, err, 512)
    check(rc, err)


def positions_to_symbols(beta, moves):
    b = np.asarray(bytearray(beta), dtype=np.uint8)
    flat = np.asarray([v for m in moves for v in m] or [0], dtype=np.int16)
    out = np.zeros(max(3, 3 * len(moves)), np.uint8)
    lib().td_positions_to_symbols(_ptr(b), len(b), _ptr(flat), len(moves), _ptr(out))
    return [tuple(int(v) for v in out[3 * d: 3 * d + 3]) for d in range(len(moves))]


def configure(warps_per_block: int, grain: int) -> None:
    if lib().td_configure(int(warps_per_block), int(grain)) != OK:
        raise TdError(INVALID_ARG, "invalid launch configuration")


def configure_steal(grain: int, split_level: int, check_every: int) -> None:
    if lib().td_configure_steal(int(grain), int(split_level), int(check_every)) != OK:
        raise TdError(INVALID_ARG, "invalid donation parameters")


def unpack_moves(row) -> list:
    return [(int(m) & 31, (int(m) >> 5) & 31, (int(m) >> 10) & 31) for m in row["moves"][: int(row["depth"])]]
