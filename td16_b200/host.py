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
