"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU baseline leg
of the benchmark load this module as the checker.  The product path
(td16_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

MAX_N = 17
MAX_DEPTH = 9
FOUND = 1
NOT_FOUND = 0
BUDGET = -2

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u8p = C.POINTER(C.c_uint8)
        L.tdo_search.argtypes = [u8p, u8p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                 C.POINTER(C.c_uint16), C.POINTER(C.c_int), C.c_void_p]
        L.tdo_search.restype = C.c_int
        L.tdo_search_batch.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.tdo_search_batch.restype = C.c_int
        L.tdo_count_odd_cycles.argtypes = [u8p, C.c_int]
        L.tdo_delta_odd_cycles.argtypes = [u8p, C.c_int, C.c_int, C.c_int]
        L.tdo_accepts.argtypes = [C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
        L.tdo_can_reach.argtypes = [C.c_int, C.c_int, C.c_float, C.c_int, C.c_int, C.c_int, C.c_int]
        L.tdo_perm_to_pair.argtypes = [C.c_void_p, C.c_int, u8p, u8p, C.POINTER(C.c_int)]
        L.tdo_positions_to_symbols.argtypes = [u8p, C.c_int, C.POINTER(C.c_uint16), C.c_int, u8p]
        L.tdo_validate.argtypes = [u8p, u8p, C.c_int, u8p, C.c_int, C.c_int, C.c_char_p, C.c_size_t]
        L.tdo_codec_key.argtypes = [u8p, C.c_int, u8p, C.c_int]
        L.tdo_codec_value.argtypes = [u8p, C.c_int, u8p, C.c_int]
        L.tdo_codec_decode_key.argtypes = [u8p, C.c_int, C.c_int, u8p]
        L.tdo_codec_decode_value.argtypes = [u8p, C.c_int, u8p, C.c_int]
        L.tdo_apply_transposition.argtypes = [u8p, C.c_int, C.c_int, C.c_int, C.c_int, u8p]
        L.tdo_compose.argtypes = [u8p, u8p, C.c_int, u8p]
        L.tdo_cycle_oneline.argtypes = [u8p, C.c_int, C.c_int, u8p]
        L.tdo_set_expansion_budget.argtypes = [C.c_uint64]
        L.tdo_set_expansion_budget.restype = None
        L.tdo_synth_perms.argtypes = [C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _u8(values, size=None):
    arr = (C.c_uint8 * (size if size is not None else max(1, len(values))))()
    for i, v in enumerate(values):
        arr[i] = int(v)
    return arr


def pack_move(i: int, j: int, k: int) -> int:
    return (i & 31) | ((j & 31) << 5) | ((k & 31) << 10)


def unpack_move(m: int):
    return (m & 31, (m >> 5) & 31, (m >> 10) & 31)


def count_odd_cycles(omega) -> int:
    return lib().tdo_count_odd_cycles(_u8(omega), len(omega))


def delta_odd_cycles(omega, a, b, c) -> int:
    return lib().tdo_delta_odd_cycles(_u8(omega), a, b, c)


def accepts(n, init_odd, min_rate, full, odd, depth) -> bool:
    return bool(lib().tdo_accepts(n, init_odd, min_rate, int(full), odd, depth))


def can_reach(n, init_odd, min_rate, max_depth, full, odd, depth) -> bool:
    return bool(lib().tdo_can_reach(n, init_odd, min_rate, max_depth, int(full), odd, depth))


def set_expansion_budget(max_expansions: int) -> None:
    """Later searches give up (status BUDGET) after this many expansions; 0 = never."""
    lib().tdo_set_expansion_budget(int(max_expansions))


def search(beta, omega, init_odd, min_rate, max_moves, full=True):
    """Single-queue reference search.  Returns (status, [(i,j,k), ...], expansions)."""
    n = len(beta)
    moves = (C.c_uint16 * MAX_DEPTH)()
    depth = C.c_int(0)

    class Stats(C.Structure):
        _fields_ = [("expansions", C.c_uint64), ("pops", C.c_uint64), ("triples", C.c_uint64)]

    st = Stats()
    rc = lib().tdo_search(_u8(beta, MAX_N), _u8(omega, MAX_N), n, int(init_odd), float(min_rate),
                          int(max_moves), int(full), moves, C.byref(depth), C.cast(C.byref(st), C.c_void_p))
    out = [unpack_move(moves[d]) for d in range(depth.value)]
    return rc, out, st.expansions


def search_batch(beta, omega, n, init_odd, min_rate, max_depth, full, threads=1):
    """Arrays: beta/omega uint8[count, 17]; the rest per instance.  Returns
    (status int32[count], depth int32[count], moves uint16[count, 9], expansions uint64[count])."""
    count = int(beta.shape[0])
    beta = np.ascontiguousarray(beta, dtype=np.uint8)
    omega = np.ascontiguousarray(omega, dtype=np.uint8)
    n = np.ascontiguousarray(n, dtype=np.uint8)
    init_odd = np.ascontiguousarray(init_odd, dtype=np.int32)
    min_rate = np.ascontiguousarray(min_rate, dtype=np.float32)
    max_depth = np.ascontiguousarray(max_depth, dtype=np.int32)
    full = np.ascontiguousarray(full, dtype=np.uint8)
    status = np.zeros(count, np.int32)
    depth = np.zeros(count, np.int32)
    moves = np.zeros((count, MAX_DEPTH), np.uint16)
    exp = np.zeros(count, np.uint64)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    rc = lib().tdo_search_batch(count, p(beta), p(omega), p(n), p(init_odd), p(min_rate), p(max_depth),
                                p(full), p(status), p(depth), p(moves), p(exp), int(threads))
    if rc != 0:
        raise ValueError("tdo_search_batch rejected its arguments")
    return status, depth, moves, exp


def synth_perms(seed: int, count: int, n_min: int, n_max: int, hard_pct: int, hard_min: int, hard_max: int):
    """The benchmark's seeded S_n instances: (perms int8[count, 16], n uint8[count])."""
    perms = np.zeros((count, 16), np.int8)
    n = np.zeros(count, np.uint8)
    rc = lib().tdo_synth_perms(C.c_uint64(seed), int(count), n_min, n_max, hard_pct, hard_min, hard_max,
                               perms.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p))
    if rc != 0:
        raise ValueError("invalid synthetic-instance parameters")
    return perms, n


def perm_to_pair(pi):
    n = len(pi)
    arr = (C.c_int8 * max(1, n))(*[int(v) for v in pi])
    beta = (C.c_uint8 * MAX_N)()
    omega = (C.c_uint8 * MAX_N)()
    init = C.c_int(0)
    lib().tdo_perm_to_pair(arr, n, beta, omega, C.byref(init))
    return list(beta[: n + 1]), list(omega[: n + 1]), init.value


def positions_to_symbols(beta, moves):
    n = len(beta)
    packed = (C.c_uint16 * max(1, len(moves)))(*[pack_move(*m) for m in moves])
    out = (C.c_uint8 * max(3, 3 * len(moves)))()
    lib().tdo_positions_to_symbols(_u8(beta, MAX_N), n, packed, len(moves), out)
    return [tuple(out[3 * m: 3 * m + 3]) for m in range(len(moves))]


def validate(beta, omega, abc_moves, max_moves):
    """Returns None when the witness replays, else the rejection message."""
    n = len(beta)
    flat = [s for mv in abc_moves for s in mv]
    err = C.create_string_buffer(256)
    rc = lib().tdo_validate(_u8(beta, MAX_N), _u8(omega, MAX_N), n, _u8(flat, max(3, len(flat))),
                            len(abc_moves), int(max_moves), err, 256)
    return None if rc == 0 else err.value.decode()


def codec_key(omega) -> bytes:
    out = (C.c_uint8 * 32)()
    ln = lib().tdo_codec_key(_u8(omega), len(omega), out, 32)
    if ln < 0:
        raise ValueError("invalid key input")
    return bytes(out[:ln])


def codec_value(abc_moves) -> bytes:
    flat = [s for mv in abc_moves for s in mv]
    out = (C.c_uint8 * 64)()
    ln = lib().tdo_codec_value(_u8(flat, max(3, len(flat))), len(abc_moves), out, 64)
    if ln < 0:
        raise ValueError("invalid value input")
    return bytes(out[:ln])


def codec_decode_key(data: bytes, n: int):
    out = (C.c_uint8 * 32)()
    rc = lib().tdo_codec_decode_key(_u8(data, max(1, len(data))), len(data), n, out)
    if rc < 0:
        raise ValueError("malformed certificate key")
    return list(out[:n])


def codec_decode_value(data: bytes):
    out = (C.c_uint8 * 96)()
    rc = lib().tdo_codec_decode_value(_u8(data, max(1, len(data))), len(data), out, 32)
    if rc < 0:
        raise ValueError("malformed certificate value")
    return [tuple(out[3 * m: 3 * m + 3]) for m in range(rc)]


def apply_transposition(cycle, a, b, c):
    n = len(cycle)
    out = (C.c_uint8 * MAX_N)()
    lib().tdo_apply_transposition(_u8(cycle, MAX_N), n, a, b, c, out)
    return list(out[:n])


def compose(p, q):
    n = len(p)
    out = (C.c_uint8 * max(1, n))()
    lib().tdo_compose(_u8(p), _u8(q), n, out)
    return list(out[:n])


def cycle_oneline(cyc, n):
    out = (C.c_uint8 * max(1, n))()
    lib().tdo_cycle_oneline(_u8(cyc), len(cyc), n, out)
    return list(out[:n])


# ---- host emulation of the engine's algorithm (libtdemu.so) -----------------
#
# Not a parity oracle: td_emu.cc restates the engine's own warp algorithm one
# lane at a time.  The CPU tests use it to check the engine's logic, and the
# benchmark's CPU baseline times the free-order algorithm with it.

EMU_PATH = os.path.join(HERE, "libtdemu.so")
EMU_INSTANCE = np.dtype([("perm", "<u8"), ("min_rate", "<f4"), ("n_symbols", "u1"), ("offset", "u1"),
                         ("max_moves", "u1"), ("packed", "u1")])
EMU_RESULT = np.dtype([("status", "<i4"), ("depth", "<i4"), ("moves", "<u2", (9,)), ("reserved", "<u2"),
                       ("expansions", "<u4")])
_emu = None


def emu():
    global _emu
    if _emu is None:
        if not os.path.exists(EMU_PATH):
            build()
        E = C.CDLL(EMU_PATH)
        E.td_emu_prepare_pair.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_int,
                                          C.c_void_p]
        E.td_emu_search_batch.argtypes = [C.c_int, C.c_void_p, C.c_uint, C.c_void_p, C.c_int]
        _emu = E
    return _emu


def emu_search_batch(beta, omega, n, init_odd, min_rate, max_depth, full, flags=0, threads=1):
    """The engine's algorithm on host threads (flags 0: free order with its
    restarts and explored-state table; 1: reference order).  Arrays as for
    search_batch.  Returns an EMU_RESULT array."""
    count = int(beta.shape[0])
    beta = np.ascontiguousarray(beta, np.uint8)
    omega = np.ascontiguousarray(omega, np.uint8)
    bc = lambda v, dt: np.broadcast_to(np.asarray(v, dt), (count,))  # noqa: E731
    n, init_odd, min_rate = bc(n, np.int32), bc(init_odd, np.int32), bc(min_rate, np.float32)
    max_depth, full = bc(max_depth, np.int32), bc(full, np.int32)
    inst = np.zeros(count, EMU_INSTANCE)
    E = emu()
    for i in range(count):
        if E.td_emu_prepare_pair(beta[i].ctypes.data, omega[i].ctypes.data, int(n[i]), int(init_odd[i]),
                                 float(min_rate[i]), int(max_depth[i]), int(full[i]),
                                 inst[i:].ctypes.data) != 0:
            raise ValueError(f"instance {i} is not a valid pair")
    res = np.zeros(count, EMU_RESULT)
    E.td_emu_search_batch(count, inst.ctypes.data, int(flags), res.ctypes.data, int(threads))
    return res
