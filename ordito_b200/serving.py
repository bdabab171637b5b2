"""Served heat-geodesic queries: a continuous-batching request loop over many resident meshes.

The serving form of ``heat_geodesic(trimesh, sources)`` (ordito/heat.py:391, with the resident
solver state of ``Trimesh.heat_solver``, ordito/mesh.py:2187): requests arrive for meshes of
different sizes; each mesh's operators and both Cholesky factors stay on the device, keyed by a
hash of its vertices and faces; a mesh is admitted only when its estimated footprint fits the HBM
budget and the device's free memory, evicting the least recently used idle meshes to make room.

Continuous batching: the scheduler thread keeps ``slots`` batches in flight, each on its own CUDA
stream. Whenever a slot frees up it takes the mesh whose oldest pending request has waited
longest, packs up to ``max_columns`` of that mesh's pending requests (one column per request: the
distance to the nearest of its sources) into one batched pass -- seeding, the two factored solves,
the gathered divergence and the shift, all on the slot's stream -- and copies the distances back
into pinned host memory. Requests that arrive while others are on the GPU join the next batch of
their mesh; batches of different meshes overlap on the device. A new mesh is set up (operators,
analysis, factorisation) on separate host threads, so the slots keep running meanwhile; its
first requests are answered at once by the unfactored path (settled CG, then the Poisson CG) before
it is factored -- the reference's rent-or-buy, which factors a system on its second solve
(ordito/heat.py:4394-4404).

Each result equals the same query run alone (``heat_geodesic_batch(mesh, [sources])``) up to the
solves' rounding: columns of a batch never mix, and the device passes are per column.
"""

from __future__ import annotations

import collections
import concurrent.futures
import ctypes
import hashlib
import math
import queue
import sys
import threading
import time
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from ordito_b200 import _lib
from ordito_b200.device import DeviceArray, PinnedArray

# Bytes a resident mesh holds per vertex, estimated before it is built: both float64 factors
# (about 140 stored values a vertex each on the path's meshes), the operators and the batch
# buffers. Replaced by the measured footprint once the mesh is set up.
ESTIMATED_BYTES_PER_VERTEX = 2 * 140 * 8 + 400
# Device memory kept free beyond the budget's accounting (allocator slack, graphs, scratch).
FREE_MEMORY_MARGIN = 2 << 30
# The interpreter's thread switch interval while a server runs: the dispatch loop retakes the GIL
# after every library call, and at the default 5 ms each retake could wait that long per busy
# setup thread (warm p99 of 150-750 ms measured, 33 ms at this value). Process-wide; restored by
# close().
SWITCH_INTERVAL = 2e-4
# How long a reading of the device's free memory is reused by admission (the margin covers it).
FREE_MEMORY_REUSE_S = 0.1
# Batch widths the passes are recorded for; a batch is padded up to the next one.
_BUCKETS = (1, 2, 4, 8, 16, 32, 64, 128)


def mesh_key(vertices: np.ndarray, faces: np.ndarray) -> str:
    """The cache key of a mesh: a BLAKE2b digest of its float32 vertices and int32 faces."""
    h = hashlib.blake2b(digest_size=16)
    v = np.ascontiguousarray(vertices, dtype=np.float32)
    f = np.ascontiguousarray(faces, dtype=np.int32)
    h.update(np.array([v.shape[0], f.size], dtype=np.int64).tobytes())
    h.update(v.tobytes())
    h.update(f.tobytes())
    return h.hexdigest()


def shard_of(key: str, world: int) -> int:
    """The rank that serves a mesh when ``world`` GPUs each run their own server (replicas: every
    mesh's requests, and its resident state, live on one GPU; no data crosses between them)."""
    return int(key[:8], 16) % max(1, world)


def bucket(k: int) -> int:
    """The recorded batch width a batch of ``k`` columns runs at."""
    for b in _BUCKETS:
        if k <= b:
            return b
    raise ValueError(f"batch of {k} columns is wider than {_BUCKETS[-1]}")


class MeshCache:
    """HBM accounting for resident meshes: a budget, reservations for meshes being set up, and
    least-recently-used eviction of idle meshes.

    Host-side bookkeeping only (no device calls): ``free_memory`` is a callable returning the
    device's free bytes, so the policy is testable without a GPU.
    """

    def __init__(self, budget: int, free_memory: Any = None, margin: int = FREE_MEMORY_MARGIN) -> None:
        self.budget = int(budget)
        self.margin = int(margin)
        self._free_memory = free_memory
        self.entries: collections.OrderedDict[str, Any] = collections.OrderedDict()
        self.sizes: dict[str, int] = {}
        self.reserved: dict[str, int] = {}
        self.evictions = 0

    @property
    def used(self) -> int:
        return sum(self.sizes.values()) + sum(self.reserved.values())

    def get(self, key: str) -> Any:
        """The resident entry (marked most recently used), or None."""
        entry = self.entries.get(key)
        if entry is not None:
            self.entries.move_to_end(key)
        return entry

    def admit(self, key: str, estimate: int, idle: Any) -> tuple[bool, list[Any]]:
        """Reserve ``estimate`` bytes for ``key``, evicting least recently used entries for which
        ``idle(entry)`` holds, oldest first, until it fits. Returns ``(reserved, evicted)``: the
        evicted entries are the caller's to release; ``reserved`` is False when the reservation
        cannot be made now (it may fit once busy meshes go idle). Raises ``MemoryError`` for a
        mesh larger than the whole budget."""
        if estimate > self.budget:
            raise MemoryError(f"mesh needs ~{estimate / 2**30:.1f} GiB, over the "
                              f"{self.budget / 2**30:.1f} GiB serving budget")
        evicted: list[Any] = []
        candidates = [k for k, e in self.entries.items() if idle(e)]
        while not self._fits(estimate) and candidates:
            victim = candidates.pop(0)
            evicted.append(self.entries.pop(victim))
            self.sizes.pop(victim, None)
            self.evictions += 1
        if not self._fits(estimate):
            return False, evicted
        self.reserved[key] = int(estimate)
        return True, evicted

    def _fits(self, estimate: int) -> bool:
        if self.used + estimate > self.budget:
            return False
        if self._free_memory is not None:
            pending = sum(self.reserved.values())
            if self._free_memory() - pending - estimate < self.margin:
                return False
        return True

    def commit(self, key: str, entry: Any, nbytes: int) -> None:
        """A reserved mesh is set up: it becomes resident at its measured size."""
        self.reserved.pop(key, None)
        self.entries[key] = entry
        self.entries.move_to_end(key)
        self.sizes[key] = int(nbytes)

    def cancel(self, key: str) -> None:
        self.reserved.pop(key, None)


@dataclass
class _Request:
    key: str
    sources: np.ndarray
    arrival: float
    future: concurrent.futures.Future
    vertices: Any = None
    faces: Any = None
    cold: bool = False  # its mesh was not resident when it arrived (it waited for a setup)


@dataclass
class _Resident:
    key: str
    mesh: Any
    solver: Any
    n: int
    nbytes: int
    d_src: DeviceArray
    d_off: DeviceArray
    h_src: PinnedArray
    h_off: PinnedArray
    d_out: DeviceArray
    pending: collections.deque = field(default_factory=collections.deque)
    busy: bool = False
    steps: dict = field(default_factory=dict)  # batch width -> recorded BatchStep

    def release(self) -> None:
        for step in self.steps.values():
            step.close()
        self.steps = {}
        self.solver.release_factorizations()
        self.mesh.release_factorizations()
        for name in ("d_src", "d_off", "d_out", "h_src", "h_off", "mesh", "solver"):
            setattr(self, name, None)


@dataclass
class _Unfactored:
    """A resident mesh whose systems are past the factorisation budget: its requests are answered
    one at a time by the unfactored path (the band march for the heat system, the mixed-precision
    multigrid solve for the Poisson system) on the setup threads, with its operators, multigrid
    hierarchy and solver states kept for the next request. ``lock`` orders them per mesh."""

    key: str
    mesh: Any
    nbytes: int
    lock: threading.Lock = field(default_factory=threading.Lock)
    pending: collections.deque = field(default_factory=collections.deque)  # always empty
    busy: bool = False
    queued: int = 0  # requests handed to the setup threads and not yet answered

    def release(self) -> None:
        with self.lock:
            if self.mesh is not None:
                self.mesh.dispose()
            self.mesh = None


@dataclass
class _Slot:
    stream: ctypes.c_void_p
    event: ctypes.c_void_p
    batch: tuple | None = None
    host: PinnedArray | None = None  # the batch's distances come back here (grown on demand)


class GeodesicServer:
    """Continuous-batching heat-geodesic service over resident meshes (see the module docstring).

    ``submit(vertices, faces, sources)`` returns a ``concurrent.futures.Future`` whose result is
    the ``(V,)`` float64 host array of distances to the nearest source; invalid sources fail the
    future with ``ValueError``, a mesh over the HBM budget with ``MemoryError``. A mesh whose
    systems are past the factorisation budget stays resident unfactored and its requests are
    answered one at a time on the setup threads (band march and multigrid). ``stats()`` reports
    request latencies (arrival to result, p50/p99), solves/s and cache behaviour.
    """

    def __init__(self, *, hbm_budget: int = 150 << 30, max_columns: int = 64, slots: int = 4,
                 max_sources: int = 32, method: str = "meshlab", setup_threads: int = 3,
                 plain_answers: int = 8, max_vertices: int = 1 << 18) -> None:
        if max_columns not in _BUCKETS:
            raise ValueError(f"max_columns must be one of {_BUCKETS}")
        self.max_columns = max_columns
        self.max_sources = max_sources
        if method != "meshlab":
            raise NotImplementedError("GeodesicServer serves method='meshlab' (its batches are the "
                                      "batched pass)")
        self.method = method
        self._switch_interval = sys.getswitchinterval()
        sys.setswitchinterval(min(self._switch_interval, SWITCH_INTERVAL))
        self._free_reading = (-1.0, 0)
        self.cache = MeshCache(hbm_budget, free_memory=self._free_memory)
        self._intake: queue.SimpleQueue = queue.SimpleQueue()
        self._setups: queue.SimpleQueue = queue.SimpleQueue()
        self._ready: queue.SimpleQueue = queue.SimpleQueue()
        self._waiting: dict[str, list[_Request]] = {}
        self._waiting_lock = threading.Lock()  # the scheduler and the setup threads share it
        self.plain_answers = plain_answers
        self._deferred: collections.deque = collections.deque()
        self._slots: list[_Slot] = []
        for _ in range(slots):
            stream, event = ctypes.c_void_p(0), ctypes.c_void_p(0)
            _lib.call("ob_stream_create", ctypes.byref(stream))
            _lib.call("ob_event_create", ctypes.byref(event))
            # The slot's pinned landing buffer, page-locked now rather than in the dispatch loop
            # (pinning ~100 MB stalls it); grown only for a mesh larger than max_vertices.
            self._slots.append(_Slot(stream, event, host=PinnedArray(max_columns * max_vertices, np.float64)))
        self._latencies: list[float] = []
        self._cold: list[bool] = []
        self._batches: list[int] = []
        self._hits = 0
        self._misses = 0
        self._first_arrival: float | None = None
        self._last_done: float | None = None
        self._running = True
        self._outstanding = 0
        self._lock = threading.Lock()
        self._idle = threading.Condition(self._lock)
        self._scheduler = threading.Thread(target=self._schedule, name="geodesic-scheduler", daemon=True)
        self._builders = [threading.Thread(target=self._build, name=f"geodesic-setup-{i}", daemon=True)
                          for i in range(max(1, setup_threads))]
        self._scheduler.start()
        for builder in self._builders:
            builder.start()

    # -- public ---------------------------------------------------------------------------------
    def submit(self, vertices: Any, faces: Any, sources: Any, *, key: str | None = None
               ) -> concurrent.futures.Future:
        future: concurrent.futures.Future = concurrent.futures.Future()
        v = np.ascontiguousarray(vertices, dtype=np.float32).reshape(-1, 3)
        f = np.ascontiguousarray(faces, dtype=np.int32).reshape(-1)
        src = np.ascontiguousarray(sources, dtype=np.int32).reshape(-1)
        n = v.shape[0]
        if src.size == 0 or src.size > self.max_sources:
            future.set_exception(ValueError(f"a request holds 1 to {self.max_sources} sources"))
            return future
        if src.min() < 0 or src.max() >= n:
            future.set_exception(ValueError(f"source index out of range [0, {n})"))
            return future
        request = _Request(key or mesh_key(v, f), src, time.perf_counter(), future, v, f)
        with self._lock:
            self._outstanding += 1
            if self._first_arrival is None:
                self._first_arrival = request.arrival
        self._intake.put(request)
        return future

    def drain(self, timeout: float | None = None) -> None:
        """Wait until every submitted request has completed."""
        with self._idle:
            self._idle.wait_for(lambda: self._outstanding == 0, timeout)

    def close(self) -> None:
        self.drain()
        self._running = False
        for _ in self._builders:
            self._setups.put(None)
        self._scheduler.join()
        for builder in self._builders:
            builder.join()
        for slot in self._slots:
            _lib.call("ob_stream_synchronize", slot.stream)
            _lib.call("ob_event_destroy", slot.event)
            _lib.call("ob_stream_destroy", slot.stream)
        self._slots = []
        for entry in list(self.cache.entries.values()):
            entry.release()
        self.cache.entries.clear()
        sys.setswitchinterval(self._switch_interval)

    def reset_stats(self) -> None:
        """Start a new measurement window (after a warm-up); the cache is kept."""
        self.drain()
        self._latencies, self._cold, self._batches = [], [], []
        self._hits = self._misses = 0
        self.cache.evictions = 0
        self._first_arrival = self._last_done = None

    def stats(self) -> dict[str, Any]:
        lat = np.array(self._latencies) * 1e3
        cold = np.array(self._cold, dtype=bool)
        span = (self._last_done - self._first_arrival) if self._latencies else 0.0

        def pct(values: np.ndarray, q: float) -> float | None:
            return float(np.percentile(values, q)) if values.size else None

        return {
            "requests": len(self._latencies),
            "solves_per_s": len(self._latencies) / span if span > 0 else None,
            "p50_ms": pct(lat, 50),
            "p99_ms": pct(lat, 99),
            "warm_requests": int((~cold).sum()) if lat.size else 0,
            "warm_p50_ms": pct(lat[~cold], 50) if lat.size else None,
            "warm_p99_ms": pct(lat[~cold], 99) if lat.size else None,
            "cold_p50_ms": pct(lat[cold], 50) if lat.size else None,
            "cold_p99_ms": pct(lat[cold], 99) if lat.size else None,
            "mean_batch": float(np.mean(self._batches)) if self._batches else None,
            "batches": len(self._batches),
            "cache_hits": self._hits,
            "cache_misses": self._misses,
            "evictions": self.cache.evictions,
            "resident_meshes": len(self.cache.entries),
            "resident_bytes": sum(self.cache.sizes.values()),
        }

    # -- scheduler thread -----------------------------------------------------------------------
    def _free_memory(self) -> int:
        now = time.perf_counter()
        if now - self._free_reading[0] > FREE_MEMORY_REUSE_S:
            free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
            _lib.call("ob_mem_info", ctypes.byref(free), ctypes.byref(total))
            self._free_reading = (now, int(free.value))
        return self._free_reading[1]

    def _schedule(self) -> None:
        while self._running or self._outstanding:
            progressed = False
            while True:
                try:
                    request = self._intake.get_nowait()
                except queue.Empty:
                    break
                self._route(request)
                progressed = True
            while True:
                try:
                    key, entry, error = self._ready.get_nowait()
                except queue.Empty:
                    break
                self._settle_setup(key, entry, error)
                progressed = True
            progressed |= self._retry_deferred()
            for slot in self._slots:
                if slot.batch is not None and self._event_done(slot.event):
                    self._finish(slot)
                    progressed = True
            for slot in self._slots:
                if slot.batch is None:
                    entry = self._next_entry()
                    if entry is None:
                        break
                    self._launch(entry, slot)
                    progressed = True
            if not progressed:
                in_flight = any(slot.batch is not None for slot in self._slots)
                time.sleep(20e-6 if in_flight else 200e-6)

    def _route(self, request: _Request) -> None:
        entry = self.cache.get(request.key)
        if entry is not None:
            self._hits += 1
            if isinstance(entry, _Unfactored):
                entry.queued += 1
                self._setups.put((entry, request))  # answered on a setup thread
            else:
                entry.pending.append(request)
            return
        request.cold = True
        with self._waiting_lock:
            if request.key in self._waiting:
                self._hits += 1  # the mesh is being set up: no second setup
                self._waiting[request.key].append(request)
                return
            self._misses += 1
            self._waiting[request.key] = [request]
        self._deferred.append(request)
        self._retry_deferred()

    def _retry_deferred(self) -> bool:
        progressed = False
        for _ in range(len(self._deferred)):
            request = self._deferred.popleft()
            estimate = ESTIMATED_BYTES_PER_VERTEX * request.vertices.shape[0]
            try:
                reserved, evicted = self.cache.admit(request.key, estimate,
                                                     lambda e: not e.busy and not e.pending
                                                     and not getattr(e, "queued", 0))
            except MemoryError as exc:
                self._fail_waiting(request.key, exc)
                progressed = True
                continue
            for victim in evicted:
                victim.release()
            if not reserved:
                self._deferred.append(request)  # retried once busy meshes go idle
                continue
            self._setups.put(request)
            progressed = True
        return progressed

    def _settle_setup(self, key: str, entry: _Resident | None, error: BaseException | None) -> None:
        with self._waiting_lock:
            waiting = self._waiting.pop(key, [])
        if error is not None:
            self.cache.cancel(key)
            for request in waiting:
                self._complete(request, error=error)
            return
        self.cache.commit(key, entry, entry.nbytes)
        if isinstance(entry, _Unfactored):
            for request in waiting:
                entry.queued += 1
                self._setups.put((entry, request))
        else:
            entry.pending.extend(waiting)

    def _fail_waiting(self, key: str, error: BaseException) -> None:
        with self._waiting_lock:
            waiting = self._waiting.pop(key, [])
        for request in waiting:
            self._complete(request, error=error)

    def _next_entry(self) -> _Resident | None:
        best, best_arrival = None, math.inf
        for entry in self.cache.entries.values():
            if not entry.busy and entry.pending and entry.pending[0].arrival < best_arrival:
                best, best_arrival = entry, entry.pending[0].arrival
        return best

    @staticmethod
    def _event_done(event: ctypes.c_void_p) -> bool:
        done = ctypes.c_int(0)
        _lib.call("ob_event_query", event, ctypes.byref(done))
        return bool(done.value)

    def _launch(self, entry: _Resident, slot: _Slot) -> None:
        requests = [entry.pending.popleft() for _ in range(min(self.max_columns, len(entry.pending)))]
        k = len(requests)
        kb = bucket(k)
        sets = [r.sources for r in requests] + [requests[-1].sources] * (kb - k)
        sizes = np.array([s.size for s in sets], dtype=np.int32)
        offsets = np.zeros(kb + 1, dtype=np.int32)
        np.cumsum(sizes, out=offsets[1:])
        total = int(offsets[-1])
        entry.h_src.array[:total] = np.concatenate(sets)
        entry.h_off.array[: kb + 1] = offsets
        st = slot.stream
        _lib.call("ob_memcpy", entry.d_src.ptr, entry.h_src.ptr, 4 * total, 0, st, 0)
        _lib.call("ob_memcpy", entry.d_off.ptr, entry.h_off.ptr, 4 * (kb + 1), 0, st, 0)
        entry.steps[kb].launch(st)  # the whole pass: one graph replay
        need = k * entry.n
        if slot.host is None or slot.host.array.size < need:
            slot.host = PinnedArray(max(need, self.max_columns * entry.n), np.float64)
        _lib.call("ob_memcpy", slot.host.ptr, entry.d_out.ptr, 8 * need, 1, st, 0)
        _lib.call("ob_event_record", slot.event, st)
        entry.busy = True
        slot.batch = (entry, requests)
        self._batches.append(k)

    def _finish(self, slot: _Slot) -> None:
        entry, requests = slot.batch
        slot.batch = None
        rows = slot.host.array
        n = entry.n
        for c, request in enumerate(requests):
            self._complete(request, result=rows[c * n:(c + 1) * n].copy())
        entry.busy = False

    def _complete(self, request: _Request, result: Any = None, error: BaseException | None = None) -> None:
        done = time.perf_counter()
        if error is not None:
            request.future.set_exception(error)
        else:
            request.future.set_result(result)
            self._latencies.append(done - request.arrival)
            self._cold.append(request.cold)
            self._last_done = done
        with self._idle:
            self._outstanding -= 1
            if self._outstanding == 0:
                self._idle.notify_all()

    # -- setup thread ---------------------------------------------------------------------------
    def _build(self) -> None:
        from ordito_b200.mesh import Trimesh  # noqa: PLC0415

        capture = ctypes.c_void_p(0)
        _lib.call("ob_stream_create", ctypes.byref(capture))
        while True:
            request = self._setups.get()
            if request is None:
                _lib.call("ob_stream_destroy", capture)
                return
            if isinstance(request, tuple):
                self._answer_unfactored(*request)
                continue
            try:
                mesh = Trimesh(request.vertices, request.faces)
                solver = mesh.heat_solver(None, method=self.method)
                solver.factor_on_second_solve = False
                self._answer_plain(request.key, mesh)
                if not solver.factor():
                    # Past the factorisation budget: kept resident, answered unfactored.
                    unfactored = _Unfactored(request.key, mesh, int(mesh.nbytes))
                    self._ready.put((request.key, unfactored, None))
                    continue
                n = mesh.n_vertices
                mesh.corner_tiles  # built now, not on the first batch
                cap_sources = self.max_columns * 2 * self.max_sources
                # The widest first: the factors' work buffers are then allocated once.
                solver.heat_factor.work(self.max_columns)
                solver.poisson_factor.work(self.max_columns)
                entry = _Resident(
                    key=request.key, mesh=mesh, solver=solver, n=n, nbytes=0,
                    d_src=DeviceArray.empty(cap_sources, np.int32),
                    d_off=DeviceArray.empty(self.max_columns + 1, np.int32),
                    h_src=PinnedArray(cap_sources, np.int32),
                    h_off=PinnedArray(self.max_columns + 1, np.int32),
                    d_out=DeviceArray.empty((self.max_columns, n), np.float64),
                )
                # Every batch width's pass recorded now, as one graph each.
                self._record(entry, capture)
                entry.nbytes = int(mesh.nbytes + solver.nbytes + entry.d_out.nbytes)
                _lib.call("ob_stream_synchronize", None)
                _lib.call("ob_stream_synchronize", capture)
                self._ready.put((request.key, entry, None))
            except BaseException as exc:  # noqa: BLE001 -- the error belongs to the requests
                self._ready.put((request.key, None, exc))

    def _answer_unfactored(self, entry: _Unfactored, request: _Request) -> None:
        from ordito_b200 import heat as gheat  # noqa: PLC0415

        with entry.lock:
            try:
                if entry.mesh is None:
                    raise RuntimeError("the mesh was evicted before its request ran")
                distances = gheat.heat_geodesic(entry.mesh, request.sources, method=self.method).numpy()
            except Exception as exc:  # noqa: BLE001 -- the error belongs to the request
                self._complete(request, error=exc)
            else:
                self._complete(request, result=distances)
            finally:
                entry.queued -= 1

    def _answer_plain(self, key: str, mesh: Any) -> None:
        """Answer up to ``plain_answers`` of the mesh's waiting requests by the unfactored path
        (rent before buy); the rest wait for the factored batches."""
        from ordito_b200 import heat as gheat  # noqa: PLC0415

        answered = 0
        while answered < self.plain_answers:
            with self._waiting_lock:
                waiting = self._waiting.get(key)
                if not waiting:
                    return
                take = waiting[: self.plain_answers - answered]
                del waiting[: len(take)]
            for request in take:
                try:
                    distances = gheat.heat_geodesic(mesh, request.sources, method=self.method).numpy()
                except Exception as exc:  # noqa: BLE001 -- the error belongs to the request
                    self._complete(request, error=exc)
                else:
                    self._complete(request, result=distances)
                answered += 1

    def _record(self, entry: _Resident, capture: ctypes.c_void_p) -> None:
        from ordito_b200 import heat as gheat  # noqa: PLC0415

        for width in reversed(_BUCKETS):
            if width > self.max_columns:
                continue
            # Valid sources for the recording runs (vertex 0 in every column).
            entry.h_src.array[:width] = 0
            entry.h_off.array[: width + 1] = np.arange(width + 1, dtype=np.int32)
            _lib.call("ob_memcpy", entry.d_src.ptr, entry.h_src.ptr, 4 * width, 0, None, 1)
            _lib.call("ob_memcpy", entry.d_off.ptr, entry.h_off.ptr, 4 * (width + 1), 0, None, 1)
            out = DeviceArray(entry.d_out.ptr, (width, entry.n), np.float64, owned=False, base=entry.d_out)
            src = DeviceArray(entry.d_src.ptr, (width,), np.int32, owned=False, base=entry.d_src)
            off = DeviceArray(entry.d_off.ptr, (width + 1,), np.int32, owned=False, base=entry.d_off)
            # The widest first runs the pass once to prepare the mesh; the rest record directly.
            entry.steps[width] = gheat.BatchStep(entry.mesh, entry.solver, src, off, width, out,
                                                 capture, warm=not entry.steps)


# -- synthetic serving workload ---------------------------------------------------------------

@dataclass
class WorkloadRequest:
    """One request of a synthetic stream: when it arrives (seconds from the start), which mesh
    (``("icosphere", level, seed)`` or ``("torus", cols, rows, seed)``) and its sources."""

    arrival: float
    mesh: tuple
    n_vertices: int
    sources: np.ndarray


def mesh_for(spec: tuple) -> tuple[np.ndarray, np.ndarray]:
    """Vertices and faces of a workload mesh spec."""
    from ordito_b200 import creation  # noqa: PLC0415

    if spec[0] == "icosphere":
        v, f = creation.icosphere(int(spec[1]))
        v = creation.radial_noise(v, 0.01, int(spec[2]))
    else:
        _, cols, rows, seed = spec
        v, f = creation.jittered_torus(int(cols), int(rows), seed=int(seed))
    return np.ascontiguousarray(v, np.float32), np.ascontiguousarray(f, np.int32)


def _spec_vertices(spec: tuple) -> int:
    if spec[0] == "icosphere":
        return 10 * 4 ** int(spec[1]) + 2
    return int(spec[1]) * int(spec[2])


def serving_workload(seed: int, n_requests: int, rate: float, *, v_min: float = 1e3,
                     v_max: float = 2e6, reuse: float = 0.7, pool: int = 50,
                     max_sources: int = 32) -> list[WorkloadRequest]:
    """A stream of heat-geodesic requests: Poisson arrivals at ``rate`` per second; each mesh's
    vertex count log-uniform in ``[v_min, v_max]`` (an icosphere at the nearest subdivision level
    with its radius perturbed by 1 % seeded noise, so a new draw is a new mesh, or a jittered
    torus with cols = 2 rows); ``reuse`` of the requests draw one of the last
    ``pool`` distinct meshes seen (cache hits for a server); 1 to ``max_sources`` uniform
    sources per request."""
    rng = np.random.default_rng(seed)
    seen: list[tuple] = []
    out: list[WorkloadRequest] = []
    clock = 0.0
    for _ in range(n_requests):
        clock += float(rng.exponential(1.0 / rate))
        if seen and rng.random() < reuse:
            spec = seen[int(rng.integers(len(seen)))]
        else:
            target = math.exp(rng.uniform(math.log(v_min), math.log(v_max)))
            if rng.random() < 0.5:
                level = int(np.clip(round(math.log((target - 2) / 10, 4)), 1, 9))
                spec = ("icosphere", level, int(rng.integers(1 << 30)))
            else:
                rows = max(4, int(round(math.sqrt(target / 2))))
                spec = ("torus", 2 * rows, rows, int(rng.integers(1 << 30)))
            if spec in seen:
                seen.remove(spec)
            seen.append(spec)
            if len(seen) > pool:
                seen.pop(0)
        n = _spec_vertices(spec)
        count = int(rng.integers(1, max_sources + 1))
        sources = rng.choice(n, size=min(count, n), replace=False).astype(np.int32)
        out.append(WorkloadRequest(clock, spec, n, sources))
    return out
