"""Host-side slot and queue model over the C ABI.

Mirrors the reference's Java host for the witness search
(emitter/src/main/java/br/unb/cic/tdp/base/GPUSortingSearch.java,
GpuDeviceLayout.java, GpuSearchStats.java): a bounded pending queue of
capacity slots + queue_capacity, one worker thread per slot blocking in the
native search, and position -> symbol conversion of the witness.  Latency
percentiles are an addition (the reference reports none).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import queue
import threading
import time
from dataclasses import dataclass

import numpy as np

from . import _lib


class GpuDeviceLayout:
    """Equal-capacity mapping of slots to CUDA devices (GpuDeviceLayout.java:15-96)."""

    def __init__(self, devices, slots_per_device: int):
        if devices is None or len(devices) == 0:
            raise ValueError("devices must contain at least one CUDA device ordinal")
        if slots_per_device <= 0:
            raise ValueError("slotsPerDevice must be positive")
        seen = set()
        for d in devices:
            if d < 0:
                raise ValueError("devices must contain only non-negative CUDA device ordinals")
            if d in seen:
                raise ValueError(f"devices must contain distinct CUDA device ordinals; duplicate: {d}")
            seen.add(d)
        total = len(devices) * slots_per_device
        if total > 2**31 - 1:
            raise ValueError("total GPU slot count is too large")
        self._devices = list(devices)
        self.slots_per_device = slots_per_device
        self.total_slots = total

    @staticmethod
    def parse_devices(value: str):
        if value is None or not value.strip():
            raise ValueError("GPU device list must not be blank")
        out = []
        for tok in value.split(","):
            tok = tok.strip()
            if not tok:
                raise ValueError("GPU device list contains an empty ordinal")
            try:
                out.append(int(tok))
            except ValueError as e:
                raise ValueError(f"GPU device list contains a non-integer ordinal: {value}") from e
        return out

    def devices(self):
        return list(self._devices)

    def device_count(self) -> int:
        return len(self._devices)

    def _check(self, slot: int):
        if slot < 0 or slot >= self.total_slots:
            raise ValueError(f"GPU slot is outside the configured range: {slot}")

    def device_for_slot(self, slot: int) -> int:
        self._check(slot)
        return self._devices[slot % len(self._devices)]

    def device_index_for_slot(self, slot: int) -> int:
        self._check(slot)
        return slot % len(self._devices)


@dataclass
class DeviceSnapshot:
    device: int
    started: int
    completed: int
    failed: int
    queue_wait_nanos: int
    busy_nanos: int


@dataclass
class Snapshot:
    elapsed_nanos: int
    started: int
    completed: int
    failed: int
    queue_wait_nanos: int
    busy_nanos: int
    total_slots: int
    devices: list
    latency_p50_ms: float = 0.0
    latency_p99_ms: float = 0.0
    latency_p999_ms: float = 0.0


class GpuSearchStats:
    """Windowed slot statistics (GpuSearchStats.java:44-131) plus latency
    percentiles over the window's completed searches (queue wait + search)."""

    def __init__(self, layout: GpuDeviceLayout, started_nanos: int):
        self.layout = layout
        self._lock = threading.Lock()
        self._window_start = started_nanos
        n = layout.device_count()
        self._active = [-1] * layout.total_slots
        self._queued = [0] * layout.total_slots
        self._started = [0] * n
        self._completed = [0] * n
        self._failed = [0] * n
        self._wait = [0] * n
        self._busy = [0] * n
        self._lat = []

    def acquired(self, slot: int, queued_at: int, acquired_at: int):
        with self._lock:
            if self._active[slot] >= 0:
                raise RuntimeError(f"GPU slot {slot} was acquired while already active")
            d = self.layout.device_index_for_slot(slot)
            self._started[d] += 1
            self._wait[d] += max(0, acquired_at - queued_at)
            self._active[slot] = acquired_at
            self._queued[slot] = queued_at

    def released(self, slot: int, released_at: int, failed: bool):
        with self._lock:
            since = self._active[slot]
            if since < 0:
                raise RuntimeError(f"GPU slot {slot} was released while inactive")
            d = self.layout.device_index_for_slot(slot)
            self._busy[d] += max(0, released_at - since)
            self._completed[d] += 1
            if failed:
                self._failed[d] += 1
            self._lat.append(max(0, released_at - self._queued[slot]))
            self._active[slot] = -1

    def snapshot(self, now: int) -> Snapshot:
        with self._lock:
            elapsed = max(1, now - self._window_start)
            for slot, since in enumerate(self._active):
                if since >= 0:
                    d = self.layout.device_index_for_slot(slot)
                    self._busy[d] += max(0, now - since)
                    self._active[slot] = now
            devs = [DeviceSnapshot(dev, self._started[i], self._completed[i], self._failed[i],
                                   self._wait[i], self._busy[i]) for i, dev in enumerate(self.layout.devices())]
            lat = np.asarray(self._lat, dtype=np.float64) / 1e6
            pct = (np.percentile(lat, [50, 99, 99.9]) if len(lat) else np.zeros(3))
            snap = Snapshot(elapsed, sum(self._started), sum(self._completed), sum(self._failed),
                            sum(self._wait), sum(self._busy), self.layout.total_slots, devs,
                            float(pct[0]), float(pct[1]), float(pct[2]))
            n = len(self._started)
            self._started, self._completed, self._failed = [0] * n, [0] * n, [0] * n
            self._wait, self._busy = [0] * n, [0] * n
            self._lat = []
            self._window_start = now
            return snap


@dataclass
class _Job:
    beta: bytes
    omega: bytes
    initial_even_cycles: int
    min_rate: float
    max_moves: int
    full_sorting: bool
    queued_at: int
    future: cf.Future


def _queue_capacity_from_env() -> int:
    v = os.environ.get("TDP_GPU_QUEUE_CAPACITY", "").strip()
    cap = int(v) if v else 0
    if cap < 0:
        raise ValueError("tdp.gpuQueueCapacity must not be negative")
    return cap


class GPUSortingSearch:
    """Singleton slot/queue front end (GPUSortingSearch.java:40-240)."""

    _instance = None
    _lock = threading.Lock()

    def __init__(self, devices, slots_per_device: int, queue_bytes_budget: int, queue_capacity: int | None = None,
                 collect_stats: bool = True):
        if queue_bytes_budget <= 0:
            raise ValueError("queueBytesBudget must be positive")
        self.layout = GpuDeviceLayout(devices, slots_per_device)
        self.total_slots = self.layout.total_slots
        self.queue_capacity = _queue_capacity_from_env() if queue_capacity is None else int(queue_capacity)
        if self.queue_capacity < 0:
            raise ValueError("tdp.gpuQueueCapacity must not be negative")
        self.pending_capacity = self.total_slots + self.queue_capacity
        self._pending: queue.Queue = queue.Queue(maxsize=self.pending_capacity)
        self.stats = GpuSearchStats(self.layout, time.monotonic_ns()) if collect_stats else None
        _lib.init_slots(self.total_slots, self.layout.devices(), queue_bytes_budget)
        self._stop = threading.Event()
        self._threads = []
        for slot in range(self.total_slots):
            t = threading.Thread(target=self._run_slot, args=(slot,), daemon=True,
                                 name=f"gpu-device-{self.layout.device_for_slot(slot)}-slot-{slot}")
            t.start()
            self._threads.append(t)

    @classmethod
    def init(cls, devices, slots_per_device: int, queue_bytes_budget: int, **kw) -> None:
        """First initialisation wins; later calls are ignored."""
        with cls._lock:
            if cls._instance is None:
                cls._instance = cls(devices, slots_per_device, queue_bytes_budget, **kw)

    @classmethod
    def get_instance(cls) -> "GPUSortingSearch":
        if cls._instance is None:
            raise RuntimeError("GPUSortingSearch has not been initialized. Call init() first.")
        return cls._instance

    @classmethod
    def shutdown(cls) -> None:
        with cls._lock:
            inst = cls._instance
            cls._instance = None
        if inst is not None:
            inst._stop.set()
            for _ in inst._threads:
                try:
                    inst._pending.put_nowait(None)
                except queue.Full:
                    pass
            for t in inst._threads:
                t.join(timeout=10)
            _lib.destroy()

    def _run_slot(self, slot: int) -> None:
        while not self._stop.is_set():
            job = self._pending.get()
            if job is None:
                return
            failed = True
            if self.stats is not None:
                self.stats.acquired(slot, job.queued_at, time.monotonic_ns())
            try:
                res = _lib.search(slot, job.beta, job.omega, job.initial_even_cycles, job.min_rate,
                                  job.max_moves, job.full_sorting)
                failed = False
                job.future.set_result(res)
            except BaseException as e:  # noqa: BLE001 - delivered to the caller's future
                job.future.set_exception(e)
            finally:
                if self.stats is not None:
                    self.stats.released(slot, time.monotonic_ns(), failed)

    def search(self, beta: bytes, omega: bytes, initial_even_cycles: int, min_rate: float, max_moves: int,
               full_sorting: bool = True):
        """Blocking search; returns the witness as symbol triples (a, b, c) on
        the caller's beta (GPUSortingSearch.java:204-240), or []."""
        fut: cf.Future = cf.Future()
        self._pending.put(_Job(bytes(beta), bytes(omega), int(initial_even_cycles), float(min_rate),
                               int(max_moves), bool(full_sorting), time.monotonic_ns(), fut))
        positions = fut.result()
        if not positions:
            return []
        return _lib.positions_to_symbols(beta, positions)


def positions_to_symbols_batch(beta: np.ndarray, depth: np.ndarray, moves: np.ndarray) -> np.ndarray:
    """Position triples -> symbol triples for a whole batch at once
    (GPUSortingSearch.java:229-238 per pair): beta uint8[c, 17], depth
    int[c], moves int16[c, 9, 3]; returns uint8[c, 9, 3] (rows past a pair's
    depth are zero)."""
    cur = np.array(beta, dtype=np.int16)
    c, width = cur.shape
    out = np.zeros((c, 9, 3), np.uint8)
    rows = np.arange(c)
    m = np.arange(width, dtype=np.int16)[None, :]
    for d in range(int(depth.max()) if c else 0):
        live = depth > d
        i, j, k = (moves[:, d, q].astype(np.int16)[:, None] for q in range(3))
        for q in range(3):
            out[live, d, q] = cur[rows[live], moves[live, d, q]]
        # block swap: positions i..k-1 take A[j..k-1] then A[i..j-1]
        inside = (m >= i) & (m < k)
        src = np.where(inside, np.where(m < i + (k - j), m + (j - i), m - (k - j)), m)
        nxt = np.take_along_axis(cur, src.astype(np.int64), axis=1)
        cur = np.where(live[:, None], nxt, cur)
    return out


class PairBatcher:
    """A case consumer that searches pairs in batches.

    The enumerator hands every canonical pair to a thread-safe
    Consumer<CyclicTargetPair> from many generator threads
    (DirectTwistedBraceletGenerator.generateRepresentativesConcurrently,
    emitter/src/main/java/br/unb/cic/tdp/DirectTwistedBraceletGenerator.java:105-156),
    and the consumer makes one blocking search per pair through the slot queue
    (GPUSortingSearch.java:134-162).  This consumer collects the pairs instead:
    a batch is handed to a slot worker when it holds `batch_size` pairs or
    when its oldest pair has waited `max_delay_s`, and the worker searches it
    with one td_search_pairs call.  `accept` returns a future of the witness
    as symbol triples (a, b, c) on the pair's beta, [] when there is none; the
    optional `sink(beta, omega, witness)` receives every found witness (e.g. a
    certificate writer), and the optional `batch_sink(beta, omega, n, status,
    depth, moves)` each searched batch as arrays (position triples).  At most `max_pending` batches wait for a worker;
    `accept` blocks beyond that, like the reference's bounded queue of
    slots + tdp.gpuQueueCapacity jobs.  `search_fn` replaces the engine call
    (the CPU tests use it)."""

    def __init__(self, slots, batch_size: int = 4096, max_delay_s: float = 0.002, max_pending: int | None = None,
                 sink=None, search_fn=None, batch_sink=None):
        self.slots = list(slots)
        if not self.slots or batch_size <= 0 or max_delay_s <= 0:
            raise ValueError("a batcher needs slots, a positive batch size and a positive delay")
        self.batch_size = int(batch_size)
        self.max_delay_s = float(max_delay_s)
        self.sink = sink
        self.batch_sink = batch_sink
        self._search = search_fn or _lib.search_pairs
        self._cv = threading.Condition()
        self._open: list = []          # (beta, omega, init, rate, maxd, full, future) of the filling batch
        self._opened_at = 0.0
        self._ready: list = []         # full or expired batches
        self._max_pending = max_pending or 2 * len(self.slots)
        self._closed = False
        self.batches = 0
        self.pairs = 0
        self._threads = [threading.Thread(target=self._work, args=(s,), daemon=True, name=f"pair-batcher-slot-{s}")
                         for s in self.slots]
        self._timer = threading.Thread(target=self._tick, daemon=True, name="pair-batcher-timer")
        for t in self._threads:
            t.start()
        self._timer.start()

    def accept(self, beta, omega, initial_even_cycles: int, min_rate: float, max_moves: int,
               full_sorting: bool = True) -> cf.Future:
        fut: cf.Future = cf.Future()
        beta, omega = bytes(beta), bytes(omega)
        if len(beta) != len(omega):
            fut.set_exception(_lib.TdError(_lib.INVALID_ARG, "beta and omega must have equal lengths"))
            return fut
        with self._cv:
            if self._closed:
                raise RuntimeError("the batcher is closed")
            while len(self._ready) >= self._max_pending:
                self._cv.wait()
            if not self._open:
                self._opened_at = time.monotonic()
            self._open.append((beta, omega, int(initial_even_cycles), float(min_rate), int(max_moves),
                               bool(full_sorting), fut))
            if len(self._open) >= self.batch_size:
                self._ready.append(self._open)
                self._open = []
                self._cv.notify_all()
        return fut

    def _tick(self):
        with self._cv:
            while not self._closed:
                if self._open and time.monotonic() - self._opened_at >= self.max_delay_s:
                    self._ready.append(self._open)
                    self._open = []
                    self._cv.notify_all()
                self._cv.wait(timeout=self.max_delay_s / 2)

    def _work(self, slot: int):
        while True:
            with self._cv:
                while not self._ready and not self._closed:
                    self._cv.wait()
                if not self._ready:
                    return
                batch = self._ready.pop(0)
                self._cv.notify_all()
            self._run(slot, batch)

    def _run(self, slot: int, batch):
        c = len(batch)
        beta = np.zeros((c, 17), np.uint8)
        omega = np.zeros((c, 17), np.uint8)
        n = np.zeros(c, np.uint8)
        for i, p in enumerate(batch):
            k = min(len(p[0]), 17)
            beta[i, :k] = np.frombuffer(p[0][:k], np.uint8)
            omega[i, :k] = np.frombuffer(p[1][:k], np.uint8)
            n[i] = len(p[0]) if len(p[0]) <= 17 else 255
        cols = [np.array([p[f] for p in batch], dt) for f, dt in ((2, np.int32), (3, np.float32), (4, np.int32),
                                                                   (5, np.uint8))]
        try:
            status, depth, moves = self._search(slot, beta, omega, n, *cols)
        except BaseException as e:  # noqa: BLE001 - delivered to every caller in the batch
            for p in batch:
                p[6].set_exception(e)
            return
        messages = {_lib.OVERFLOW: "GPU sorting search queue overflow",
                    _lib.TIMEOUT: "GPU sorting search deadline reached",
                    _lib.INVALID_ARG: "performGpuSortingSearch: invalid input"}
        depth = np.where(status == _lib.OK, depth, 0)
        symbols = positions_to_symbols_batch(beta, depth, moves)
        if self.batch_sink is not None:
            self.batch_sink(beta, omega, n, status, depth, moves)
        for i, p in enumerate(batch):
            st = int(status[i])
            if st == _lib.OK:
                witness = [tuple(int(v) for v in symbols[i, d]) for d in range(int(depth[i]))]
                if self.sink is not None:
                    self.sink(p[0], p[1], witness)
                p[6].set_result(witness)
            elif st == _lib.NOT_FOUND:
                p[6].set_result([])
            else:
                p[6].set_exception(_lib.TdError(st, messages.get(st, "GPU sorting search failed")))
        with self._cv:
            self.batches += 1
            self.pairs += c

    def close(self) -> None:
        """Searches what was accepted, then stops the workers."""
        with self._cv:
            if self._open:
                self._ready.append(self._open)
                self._open = []
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        self._timer.join()
