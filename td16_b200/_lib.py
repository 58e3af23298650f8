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
                ("donations", C.c_uint64), ("donated_items", C.c_uint64), ("races", C.c_uint64)]


class ServeStats(C.Structure):
    _fields_ = [("p50_ms", C.c_double), ("p99_ms", C.c_double), ("p999_ms", C.c_double), ("mean_ms", C.c_double),
                ("max_ms", C.c_double), ("offered_per_s", C.c_double), ("served_per_s", C.c_double),
                ("wall_s", C.c_double), ("admission_wait_ms_mean", C.c_double), ("served", C.c_uint64),
                ("found", C.c_uint64), ("workers", C.c_int), ("max_inflight", C.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class BatcherStats(C.Structure):
    _fields_ = [(name, C.c_uint64) for name in ("pairs", "batches", "found", "not_found", "errors",
                                                 "certificates")] + [("search_s", C.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# td_batcher_done_fn: (user, count, tags, status, depth, out_ijk)
BATCHER_DONE = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_int32),
                           C.POINTER(C.c_int32), C.POINTER(C.c_int16))


# td_batcher_search_fn: td_search_pairs' signature
BATCHER_SEARCH = C.CFUNCTYPE(C.c_int, C.c_int, C.c_int, *([C.c_void_p] * 7), C.c_uint, *([C.c_void_p] * 3),
                             C.c_void_p, C.c_size_t)


class TdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None

EXPORTS = ["td_init_slots", "td_search", "td_search_ordered", "td_slot_count", "td_slot_device",
           "td_slot_stream", "td_destroy", "td_prepare_pairs", "td_prepare_perms", "td_synth_perms",
           "td_search_batch", "td_search_batch_device", "td_validate_batch_device",
           "td_positions_to_symbols", "td_configure", "td_configure_steal", "td_configure_serve", "td_configure_table", "td_configure_restart", "td_configure_race",
           "td_set_time_limit", "td_int_issue_peak",
           "td_codec_key", "td_codec_value", "td_codec_decode_key", "td_codec_decode_value",
           "td_replay_symbols_device", "td_cert_writer_open", "td_cert_writer_enqueue", "td_cert_writer_close",
           "td_serve_open", "td_serve_workers", "td_serve_submit", "td_serve_poll", "td_serve_close",
           "td_serve_open_loop", "td_configure_percall", "td_search_pairs", "td_percall_open_loop", "td_cert_writer_enqueue_batch", "td_cert_read_file", "td_pairs_from_perms", "td_batch_graph_create", "td_batch_graph_launch", "td_batch_graph_destroy",
           "td_batcher_open", "td_batcher_accept", "td_batcher_flush", "td_batcher_close", "td_configure_split"]


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
    L.td_configure_serve.argtypes = [C.c_int, C.c_int, C.c_int]
    L.td_configure_table.argtypes = [C.c_int]
    L.td_configure_restart.argtypes = [C.c_int]
    L.td_configure_race.argtypes = [C.c_int]
    L.td_configure_split.argtypes = [C.c_int, C.c_int]
    L.td_set_time_limit.argtypes = [C.c_double]
    L.td_configure_percall.argtypes = [C.c_int, C.c_double, C.c_double]
    L.td_percall_open_loop.argtypes = [C.c_int, vp, C.c_int, C.c_double, C.c_uint64, C.c_int, vp,
                                       C.POINTER(ServeStats), cp, sz]
    L.td_search_pairs.argtypes = [C.c_int, C.c_int] + [vp] * 7 + [C.c_uint] + [vp] * 3 + [cp, sz]
    L.td_codec_key.argtypes = [vp, C.c_int, vp, C.c_int]
    L.td_codec_value.argtypes = [vp, C.c_int, vp, C.c_int]
    L.td_codec_decode_key.argtypes = [vp, C.c_int, C.c_int, vp]
    L.td_codec_decode_value.argtypes = [vp, C.c_int, vp, C.c_int]
    L.td_replay_symbols_device.argtypes = [C.c_int, vp, vp, vp, vp, vp, vp, vp, vp, cp, sz]
    L.td_cert_writer_open.argtypes = [cp, C.c_double]
    L.td_cert_writer_open.restype = vp
    L.td_cert_writer_enqueue.argtypes = [vp, vp, C.c_int, vp, C.c_int]
    L.td_cert_writer_close.argtypes = [vp]
    L.td_cert_writer_close.restype = C.c_longlong
    L.td_batch_graph_create.argtypes = [C.c_int, C.c_int, vp, vp, C.c_uint, C.c_uint64, C.POINTER(vp), cp, sz]
    L.td_batch_graph_launch.argtypes = [vp, vp, cp, sz]
    L.td_batch_graph_destroy.argtypes = [vp]
    L.td_cert_writer_enqueue_batch.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.td_cert_writer_enqueue_batch.restype = C.c_longlong
    L.td_cert_read_file.argtypes = [cp, C.c_int, C.c_longlong, vp, vp, vp]
    L.td_cert_read_file.restype = C.c_longlong
    L.td_pairs_from_perms.argtypes = [C.c_int, vp, vp, vp, vp]
    L.td_pairs_from_perms.restype = None
    L.td_serve_open.argtypes = [C.c_int, C.c_uint, C.c_uint, C.c_double, C.POINTER(vp), cp, sz]
    L.td_serve_workers.argtypes = [vp]
    L.td_serve_submit.argtypes = [vp, vp, C.POINTER(C.c_ulonglong)]
    L.td_serve_poll.argtypes = [vp, C.c_ulonglong, vp]
    L.td_serve_close.argtypes = [vp, cp, sz]
    L.td_serve_open_loop.argtypes = [C.c_int, vp, C.c_int, C.c_double, C.c_uint64, C.c_uint64, C.c_uint, vp,
                                     C.POINTER(ServeStats), cp, sz]
    L.td_batcher_open.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint, BATCHER_SEARCH, vp,
                                  BATCHER_DONE, vp, C.POINTER(vp), cp, sz]
    L.td_batcher_accept.argtypes = [vp, C.c_uint64, vp, vp, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int]
    L.td_batcher_flush.argtypes = [vp]
    L.td_batcher_close.argtypes = [vp, C.POINTER(BatcherStats), cp, sz]
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


def search_pairs(slot: int, beta, omega, n, init, min_rate, max_moves, full=1, ordered: bool = False):
    """Many reference pairs in one call (td_search_pairs).  beta/omega
    uint8[count, 17]; the rest per pair or broadcast.  Returns (status
    int32[count] with the per-call codes, depth int32[count], position
    triples int16[count, 9, 3])."""
    count = int(beta.shape[0])
    beta = np.ascontiguousarray(beta, np.uint8)
    omega = np.ascontiguousarray(omega, np.uint8)
    bc = lambda v, dt: np.ascontiguousarray(np.broadcast_to(v, (count,)), dt)  # noqa: E731
    arrs = [bc(n, np.uint8), bc(init, np.int32), bc(min_rate, np.float32), bc(max_moves, np.int32),
            bc(full, np.uint8)]
    status = np.zeros(count, np.int32)
    depth = np.zeros(count, np.int32)
    moves = np.zeros((count, 9, 3), np.int16)
    err = C.create_string_buffer(512)
    rc = lib().td_search_pairs(int(slot), count, _ptr(beta), _ptr(omega), *[_ptr(a) for a in arrs],
                               FLAG_ORDERED if ordered else 0, _ptr(status), _ptr(depth), _ptr(moves), err, 512)
    check(rc, err)
    return status, depth, moves


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


def search_batch(slot: int, instances: np.ndarray, flags: int = 0, max_expansions: int = 0, out=None):
    """Host arrays in and out.  Returns (results, BatchStats).  `out`, when
    given, is a contiguous RESULT_DTYPE array of the same length that receives
    the results (e.g. a view of pinned host memory, so that the copies run at
    full PCIe speed)."""
    instances = np.ascontiguousarray(instances, INSTANCE_DTYPE)
    if out is None:
        results = np.zeros(len(instances), RESULT_DTYPE)
    else:
        results = out
        if results.dtype != RESULT_DTYPE or len(results) != len(instances) or not results.flags["C_CONTIGUOUS"]:
            raise TdError(INVALID_ARG, "out must be a contiguous result array of the batch's length")
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


def set_time_limit(seconds: float) -> None:
    if lib().td_set_time_limit(float(seconds)) != OK:
        raise TdError(INVALID_ARG, "time limit must be positive")


def configure_steal(grain: int, split_level: int, check_every: int) -> None:
    if lib().td_configure_steal(int(grain), int(split_level), int(check_every)) != OK:
        raise TdError(INVALID_ARG, "invalid donation parameters")


def configure_table(bits: int) -> None:
    """Explored-state tables of the free order: 2^bits entries per warp, 0 = none."""
    if lib().td_configure_table(int(bits)) != OK:
        raise TdError(INVALID_ARG, "table bits must be 0 or 6..16")


def configure_restart(base: int) -> None:
    """Restart budgets of free-order batch searches: base x Luby sequence, 0 = none."""
    if lib().td_configure_restart(int(base)) != OK:
        raise TdError(INVALID_ARG, "restart base must be 0 or >= 16")


def configure_race(attempt: int) -> None:
    """Free-order batches: a search that starts restart attempt `attempt`
    (1..32) races a search of its inverse permutation; 0 = off.  Verdicts do
    not depend on it."""
    if lib().td_configure_race(int(attempt)) != OK:
        raise TdError(INVALID_ARG, "race attempt: 0..32")


def configure_split(first_pass_expansions: int = 64, records: int = 1 << 20) -> None:
    """Reference-order batches: one-warp first pass of `first_pass_expansions`
    (0 = no split), then walks left over split below the root into at most
    `records` subtrees per launch.  Results do not depend on either."""
    if lib().td_configure_split(int(first_pass_expansions), int(records)) != OK:
        raise TdError(INVALID_ARG, "split settings: expansions >= 0, 1 <= records <= 2^24")


def configure_percall(mode: int, rotate_after_s: float = 0.0, idle_exit_s: float = 0.0) -> None:
    """Per-call searches: 1 through the device's resident server (default),
    0 one launch per call; rotate_after_s > 0 sets the server's rotation age,
    idle_exit_s > 0 the idle time after which it exits by itself."""
    if lib().td_configure_percall(int(mode), float(rotate_after_s), float(idle_exit_s)) != OK:
        raise TdError(INVALID_ARG, "per-call mode must be 0 or 1 and the times >= 0")


def configure_serve(grain: int, split_level: int, check_every: int) -> None:
    """Work donation of later serving launches (latency-oriented defaults 1, 2, 32)."""
    if lib().td_configure_serve(int(grain), int(split_level), int(check_every)) != OK:
        raise TdError(INVALID_ARG, "invalid donation parameters")


def unpack_moves(row) -> list:
    return [(int(m) & 31, (int(m) >> 5) & 31, (int(m) >> 10) & 31) for m in row["moves"][: int(row["depth"])]]


# ---- certificate format (CertificateCodec.java) ----------------------------

def codec_key(omega) -> bytes:
    o = np.frombuffer(bytes(omega), np.uint8).copy()
    out = np.zeros(32, np.uint8)
    n = lib().td_codec_key(_ptr(o), len(o), _ptr(out), 32)
    if n < 0:
        raise TdError(INVALID_ARG, "certificate keys need 1..32 symbols below 32")
    return out[:n].tobytes()


def codec_value(abc_moves) -> bytes:
    flat = np.asarray([v for m in abc_moves for v in m] or [0], np.uint8)
    out = np.zeros(64, np.uint8)
    n = lib().td_codec_value(_ptr(flat), len(abc_moves), _ptr(out), 64)
    if n < 0:
        raise TdError(INVALID_ARG, "a certificate must contain at least one move of symbols below 32")
    return out[:n].tobytes()


def codec_decode_key(data: bytes, n: int):
    d = np.frombuffer(bytes(data) or b"\0", np.uint8).copy()
    out = np.zeros(32, np.uint8)
    if lib().td_codec_decode_key(_ptr(d), len(data), int(n), _ptr(out)) < 0:
        raise TdError(INVALID_ARG, "malformed certificate key")
    return out[:n].tolist()


def codec_decode_value(data: bytes):
    d = np.frombuffer(bytes(data) or b"\0", np.uint8).copy()
    out = np.zeros(96, np.uint8)
    k = lib().td_codec_decode_value(_ptr(d), len(data), _ptr(out), 32)
    if k < 0:
        raise TdError(INVALID_ARG, "malformed certificate value")
    return [tuple(int(v) for v in out[3 * m: 3 * m + 3]) for m in range(k)]


class CertificateWriter:
    """Batched flat-file sink of certificate records (AsyncCertificateWriter semantics)."""

    def __init__(self, path: str, flush_seconds: float = 5.0):
        self._h = lib().td_cert_writer_open(path.encode(), float(flush_seconds))
        if not self._h:
            raise TdError(INVALID_ARG, f"cannot open {path}")

    def enqueue(self, omega, abc_moves) -> None:
        o = np.frombuffer(bytes(omega), np.uint8).copy()
        flat = np.asarray([v for m in abc_moves for v in m] or [0], np.uint8)
        rc = lib().td_cert_writer_enqueue(self._h, _ptr(o), len(o), _ptr(flat), len(abc_moves))
        if rc == -2:
            raise TdError(CUDA_ERROR, "certificate writer failed")
        if rc != 0:
            raise TdError(INVALID_ARG, "unencodable certificate")

    def close(self) -> int:
        n = lib().td_cert_writer_close(self._h)
        self._h = None
        if n < 0:
            raise TdError(CUDA_ERROR, "certificate writer failed")
        return int(n)


def read_certificates(path: str):
    """Reads the flat file written by CertificateWriter: [(key, value), ...]."""
    data = open(path, "rb").read()
    out, i = [], 0
    while i < len(data):
        kl, vl = data[i], data[i + 1]
        out.append((data[i + 2: i + 2 + kl], data[i + 2 + kl: i + 2 + kl + vl]))
        i += 2 + kl + vl
    return out


# ---- serving (continuous batching) -----------------------------------------

class Server:
    """A resident serving launch: submit requests while others run."""

    def __init__(self, device: int = 0, ring_size: int = 4096, flags: int = 0, time_limit_s: float = 60.0):
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        check(lib().td_serve_open(int(device), int(ring_size), int(flags), float(time_limit_s), C.byref(h), err, 512),
              err)
        self._h = h
        self.workers = lib().td_serve_workers(h)

    def submit(self, instance) -> int:
        x = np.ascontiguousarray(np.asarray(instance, INSTANCE_DTYPE).reshape(1))
        t = C.c_ulonglong()
        rc = lib().td_serve_submit(self._h, _ptr(x), C.byref(t))
        if rc != OK:
            raise TdError(rc, "serving ring is full")
        return t.value

    def poll(self, ticket: int):
        out = np.zeros(1, RESULT_DTYPE)
        return out[0] if lib().td_serve_poll(self._h, C.c_ulonglong(ticket), _ptr(out)) else None

    def close(self) -> None:
        err = C.create_string_buffer(512)
        check(lib().td_serve_close(self._h, err, 512), err)
        self._h = None


def serve_open_loop(device: int, instances: np.ndarray, rate: float, seed: int = 3,
                    pool_bytes: int = 64 << 30, flags: int = 0):
    """Open-loop Poisson experiment; returns (results, stats dict)."""
    instances = np.ascontiguousarray(instances, INSTANCE_DTYPE)
    results = np.zeros(len(instances), RESULT_DTYPE)
    st = ServeStats()
    err = C.create_string_buffer(512)
    rc = lib().td_serve_open_loop(int(device), _ptr(instances), len(instances), float(rate), C.c_uint64(seed),
                                  C.c_uint64(pool_bytes), int(flags), _ptr(results), C.byref(st), err, 512)
    check(rc, err)
    return results, st.as_dict()


def percall_open_loop(device: int, instances: np.ndarray, rate: float, clients: int = 64, seed: int = 3):
    """Open-loop Poisson stream through the per-call server, latency measured
    by client threads that poll only their own requests; returns (results,
    stats dict)."""
    instances = np.ascontiguousarray(instances, INSTANCE_DTYPE)
    results = np.zeros(len(instances), RESULT_DTYPE)
    st = ServeStats()
    err = C.create_string_buffer(512)
    rc = lib().td_percall_open_loop(int(device), _ptr(instances), len(instances), float(rate), C.c_uint64(seed),
                                    int(clients), _ptr(results), C.byref(st), err, 512)
    check(rc, err)
    return results, st.as_dict()


class BatchGraph:
    """A captured batch launch over fixed device buffers (CUDA graph)."""

    def __init__(self, slot: int, count: int, d_instances: int, d_results: int, flags: int = 0,
                 max_expansions: int = 0):
        h = C.c_void_p()
        err = C.create_string_buffer(512)
        check(lib().td_batch_graph_create(int(slot), int(count), C.c_void_p(d_instances), C.c_void_p(d_results),
                                          int(flags), C.c_uint64(max_expansions), C.byref(h), err, 512), err)
        self._h = h

    def launch(self, stream: int | None = None) -> None:
        err = C.create_string_buffer(512)
        check(lib().td_batch_graph_launch(self._h, C.c_void_p(stream) if stream else None, err, 512), err)

    def close(self) -> None:
        if self._h:
            lib().td_batch_graph_destroy(self._h)
            self._h = None


# ---- native slot threads (td_slot_threads.cc) ---------------------------------

THREADS_PATH = os.path.join(PKG, "libtd16_slot_threads.so")
_threads = None


def _threads_lib():
    global _threads
    if _threads is None:
        if not os.path.exists(THREADS_PATH):
            raise ImportError(f"{THREADS_PATH} is missing: build it with `python -m td16_b200.build`")
        h = C.CDLL(THREADS_PATH)
        h.td_slot_threads_run.restype = C.c_double
        h.td_slot_threads_run.argtypes = [C.c_int, C.c_void_p, C.c_int] + [C.c_void_p] * 7 + [
            C.c_int, C.c_int] + [C.c_void_p] * 5
        h.td_producer_threads_run.restype = C.c_double
        h.td_producer_threads_run.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int] + [C.c_void_p] * 8
        _threads = h
    return _threads


def slot_threads_run(fn, beta, omega, n, init, rate, maxd, full, threads: int, first_slot: int = 0,
                     kind: int = 0):
    """Runs one blocking search per instance from `threads` native threads
    (thread t on slot first_slot + t), through the entry point at address
    `fn` (kind 0: td_search's signature; kind 1: the reference driver's).
    beta/omega uint8[count, 17]; the rest per instance.  Returns a dict with
    the wall time, status (1 found, 0 not found, -1 error), the entry's return
    codes, depths, position moves int16[count, 9, 3] and per-call latencies."""
    count = int(beta.shape[0])
    beta = np.ascontiguousarray(beta, np.uint8)
    omega = np.ascontiguousarray(omega, np.uint8)
    bc = lambda v, dt: np.ascontiguousarray(np.broadcast_to(v, (count,)), dt)  # noqa: E731
    n, init, rate, maxd, full = (bc(n, np.int32), bc(init, np.int32), bc(rate, np.float32), bc(maxd, np.int32),
                                 bc(full, np.uint8))
    status = np.zeros(count, np.int32)
    code = np.zeros(count, np.int32)
    depth = np.zeros(count, np.int32)
    moves = np.zeros((count, 9, 3), np.int16)
    lat = np.zeros(count, np.float64)
    secs = _threads_lib().td_slot_threads_run(int(kind), C.c_void_p(fn), count, *[_ptr(a) for a in (
        beta, omega, n, init, rate, maxd, full)], int(threads), int(first_slot),
        *[_ptr(a) for a in (status, code, depth, moves, lat)])
    return {"seconds": secs, "status": status, "code": code, "depth": depth, "moves": moves, "latency_s": lat}


def entry_address(name: str) -> int:
    """Address of an entry point of the engine library (for slot_threads_run)."""
    return C.cast(getattr(lib(), name), C.c_void_p).value


# ---- native pair consumer (td_batcher.cc) ---------------------------------------


class PairConsumer:
    """The enumerator's Consumer<CyclicTargetPair> in native code (td_batcher_*):
    producers hand pairs over one at a time with `accept`; one native worker
    per slot searches them in batches of `batch_size` (or whatever has waited
    `max_delay_s`).  Found witnesses go to `cert_writer` (a CertificateWriter)
    when given; `on_batch(tags, status, depth, moves)` receives each searched
    batch as arrays (copies) when given.  `accept` blocks while `max_pending`
    full batches wait (0: twice the slots).  `search` (a BATCHER_SEARCH
    callable) replaces td_search_pairs; the CPU tests use it."""

    def __init__(self, first_slot: int, slots: int, batch_size: int = 65536, max_delay_s: float = 0.002,
                 max_pending: int = 0, ordered: bool = False, cert_writer=None, on_batch=None, search=None):
        self._on_batch = on_batch
        self._cb = BATCHER_DONE(self._deliver) if on_batch is not None else BATCHER_DONE()
        self._search = search if search is not None else BATCHER_SEARCH()
        self._h = C.c_void_p()
        err = C.create_string_buffer(512)
        rc = lib().td_batcher_open(int(first_slot), int(slots), int(batch_size), float(max_delay_s), int(max_pending),
                                   FLAG_ORDERED if ordered else 0, self._search,
                                   cert_writer._h if cert_writer is not None else None, self._cb, None,
                                   C.byref(self._h), err, 512)
        check(rc, err)
        self.stats = None

    def _deliver(self, _user, count, tags, status, depth, ijk):
        t = np.ctypeslib.as_array(tags, (count,)).copy()
        st = np.ctypeslib.as_array(status, (count,)).copy()
        d = np.ctypeslib.as_array(depth, (count,)).copy()
        m = np.ctypeslib.as_array(ijk, (count * 27,)).reshape(count, 9, 3).copy()
        self._on_batch(t, st, d, m)

    @property
    def handle(self):
        return self._h.value

    def accept(self, tag: int, beta, omega, initial_even_cycles: int, min_rate: float, max_moves: int,
               full_sorting: bool = True) -> None:
        beta, omega = bytes(beta), bytes(omega)
        if len(beta) != len(omega):
            raise TdError(INVALID_ARG, "beta and omega must have equal lengths")
        rc = lib().td_batcher_accept(self._h, int(tag), beta, omega, len(beta), int(initial_even_cycles),
                                     float(min_rate), int(max_moves), int(bool(full_sorting)))
        check(rc, None)

    def flush(self) -> None:
        lib().td_batcher_flush(self._h)

    def close(self) -> dict:
        if self._h:
            st = BatcherStats()
            err = C.create_string_buffer(512)
            rc = lib().td_batcher_close(self._h, C.byref(st), err, 512)
            self._h = C.c_void_p()
            self.stats = st.as_dict()
            check(rc, err)
        return self.stats


def producer_threads_run(consumer: PairConsumer, threads: int, beta, omega, n, init, rate, maxd, full=1) -> float:
    """Hands `count` pairs to `consumer` from `threads` native producer threads
    (thread t: pairs t, t + threads, ..., tagged with their index).  Returns
    the producers' wall time in seconds."""
    count = int(beta.shape[0])
    beta = np.ascontiguousarray(beta, np.uint8)
    omega = np.ascontiguousarray(omega, np.uint8)
    bc = lambda v, dt: np.ascontiguousarray(np.broadcast_to(v, (count,)), dt)  # noqa: E731
    arrs = [bc(n, np.int32), bc(init, np.int32), bc(rate, np.float32), bc(maxd, np.int32), bc(full, np.uint8)]
    first = np.zeros(1, np.int32)
    secs = _threads_lib().td_producer_threads_run(C.c_void_p(entry_address("td_batcher_accept")), consumer.handle,
                                                  int(threads), count, _ptr(beta), _ptr(omega),
                                                  *[_ptr(a) for a in arrs], _ptr(first))
    if first[0] != OK:
        raise TdError(int(first[0]), f"a producer's accept returned {int(first[0])}")
    return secs
