"""Continuous-batching server for trajectory jobs (host scheduling over the C ABI).

Jobs of mixed grid, component count and mode arrive over time.  Jobs whose
configurations differ only in temperature and seed share a *bucket*: one
batched engine whose members are slots.  A job is admitted into a free slot
as soon as it has arrived and a slot (or HBM for a new bucket engine) is
free; a bucket whose slots are all free gives its HBM back when another shape
needs it.  Each bucket keeps one chunk of steps in flight on its own CUDA
stream, so buckets overlap on the device; the loop polls each chunk's event,
reads finished jobs back and reuses their slots.  A job that no empty server
could hold is refused up front (AdmissionError), so the loop never waits for
room that cannot appear.  partition_jobs / serve_distributed split a stream
over ranks (one server per GPU) with a single gather of statistics at the end.

A job's result does not depend on what else is running: its noise is keyed by
(server seed, job key) at the job's own step count (engine step index minus
the step at admission), its temperature enters as the amplitude factor
sqrt(kBT_job / kBT_engine), and members of a batch never interact.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math
import time
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import FP32, Config, Engine
from .initial import initial_state_device


@dataclasses.dataclass
class Job:
    key: int                      # unique id; keys the job's noise stream
    config: Config                # solver configuration (precision ignored; the server sets it)
    state: Optional[np.ndarray]   # initial State (reference layout, complex128), or None with `initial`
    nsteps: int
    arrival: float = 0.0          # seconds after the server starts
    initial: Optional[str] = None  # `set` lines generating the initial state on the device (when state is None)
    green_kubo: Optional[Tuple[int, int]] = None   # (nevery, nblock): Yokota-Green-Kubo stress measure
    # filled by the server
    result: Optional[np.ndarray] = None
    gk_sums: Optional[np.ndarray] = None          # [tau, mode] sums; S_mean = gk_sums / gk_blocks
    gk_blocks: int = 0
    admitted: Optional[float] = None
    finished: Optional[float] = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def bucket_key(cfg: Config, green_kubo: Optional[Tuple[int, int]] = None) -> bytes:
    """Configuration bytes with the per-job fields (temperature, seed, batch) cleared,
    plus the Green-Kubo request (one measure setting per bucket engine)."""
    c = cfg.copy()
    c.kBT = 0.0
    c.noise_seed = 0
    c.batch = 1
    c.member_offset = 0
    c.precision = 0
    return bytes(memoryview(c).cast("B")) + repr(green_kubo).encode()


_POLL_S = 5e-5  # interval of the loop's event polling while every bucket has a chunk in flight


def _noisy(cfg: Config) -> bool:
    return bool(cfg.noise_momentum or cfg.noise_order_parameter)


def _torch_event(engine):
    """A CUDA event recorded on the engine's stream after its enqueued work."""
    import torch
    ev = torch.cuda.Event()
    ev.record(torch.cuda.ExternalStream(engine.stream))
    return ev


class _Bucket:
    def __init__(self, cfg: Config, slots: int, precision: int, seed: int, graph_chunk: int = 0,
                 green_kubo: Optional[Tuple[int, int]] = None, engine_factory=Engine, autotune: int = 0):
        c = cfg.copy()
        c.batch = slots
        c.precision = precision
        c.noise_seed = seed
        c.member_offset = 0
        if _noisy(cfg):
            c.kBT = 1.0  # members carry sqrt(kBT_job) as their amplitude factor
        self.engine = engine_factory(c)
        self.device_bytes = int(self.engine.get_info().device_bytes)
        self.graph_chunk = graph_chunk
        if graph_chunk > 0:
            self.engine.set_graph_chunk(graph_chunk)
        self.autotune = autotune      # trial steps for timing the engine's kernels on its first job (0: no)
        self.green_kubo = green_kubo
        if green_kubo is not None:
            self.engine.gk_enable(*green_kubo)
        self.slots: List[Optional[Job]] = [None] * slots
        self.remaining = [0] * slots
        self.step_index = 0
        self.noisy = _noisy(cfg)
        self.inflight: Optional[Tuple[int, object]] = None   # (steps, completion event) of the enqueued chunk
        for m in range(slots):
            self.engine.set_member(m, key=0, active=False)

    def free_slot(self) -> Optional[int]:
        for m, j in enumerate(self.slots):
            if j is None:
                return m
        return None

    def admit(self, m: int, job: Job, now: float) -> None:
        if job.state is not None:
            self.engine.set_state(job.state, member=m)
        elif job.initial is not None:
            initial_state_device(self.engine, job.initial, member=m)
        else:
            raise ValueError(f"job {job.key}: neither an initial state nor `set` lines")
        scale = math.sqrt(job.config.kBT) if self.noisy else 0.0
        self.engine.set_member(m, key=job.key, step_origin=self.step_index, noise_scale=scale, active=True)
        if self.green_kubo is not None:
            self.engine.gk_read(m, reset=True)  # the slot's previous job's sums
        if self.autotune:
            # kernel family and launch shapes timed on the first job's state (state, step count and
            # measure sums restored); the server's graph chunk is kept, since staggered slots need it
            self.engine.autotune(self.autotune)
            if self.graph_chunk > 0:
                self.engine.set_graph_chunk(self.graph_chunk)
            self.autotune = 0
        self.slots[m] = job
        self.remaining[m] = job.nsteps
        job.admitted = now

    def active(self) -> bool:
        return any(j is not None for j in self.slots)


class AdmissionError(RuntimeError):
    """A job that no empty server could hold (its bucket of one slot exceeds the HBM budget)."""


class Server:
    """Continuous batching of trajectory jobs within a device-memory budget.

    `hbm_budget` caps the device bytes of the bucket engines (default: 80% of the free
    memory).  A bucket whose slots are all free is destroyed, and its bytes returned to the
    budget, when a job needs room for a new bucket.  A job that would not fit even into an
    empty server is refused with AdmissionError before anything runs.  `engine_factory`
    (default: the engine) and `event_factory` (default: a CUDA event on the engine's stream)
    are the only device-facing parts; tests of the scheduling replace them."""

    def __init__(self, precision: int = FP32, seed: int = 20240601, max_slots: int = 32, chunk: int = 25,
                 hbm_budget: Optional[int] = None, graphs: bool = True, engine_factory=Engine, event_factory=_torch_event,
                 autotune: int = 0):
        self.graphs = graphs
        self.autotune = autotune      # > 0: each new bucket engine autotunes (trials of this many steps) on its first job
        self.precision = precision
        self.seed = seed
        self.max_slots = max_slots
        self.chunk = chunk
        self.engine_factory = engine_factory
        self.event_factory = event_factory
        if hbm_budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info()
            hbm_budget = int(0.8 * free)
        self.budget = int(hbm_budget)
        self.used = 0
        self.buckets: Dict[bytes, List[_Bucket]] = {}
        self.buckets_created = 0
        self.buckets_released = 0
        self._member_bytes: Dict[bytes, int] = {}

    def _per_member_bytes(self, key: bytes, cfg: Config) -> int:
        if key not in self._member_bytes:
            c = cfg.copy()
            c.batch = 1
            c.precision = self.precision
            probe = self.engine_factory(c)
            try:
                self._member_bytes[key] = int(probe.get_info().device_bytes) + probe.info.state_doubles * 8
            finally:
                probe.close()
        return self._member_bytes[key]

    def _release_idle(self) -> int:
        """Destroy bucket engines with no job and nothing in flight; return the bytes freed."""
        freed = 0
        for key in list(self.buckets):
            keep = []
            for b in self.buckets[key]:
                if b.active() or b.inflight is not None:
                    keep.append(b)
                else:
                    b.engine.close()
                    freed += b.device_bytes
                    self.buckets_released += 1
            if keep:
                self.buckets[key] = keep
            else:
                del self.buckets[key]
        self.used -= freed
        return freed

    def _slot_for(self, job: Job) -> Optional[Tuple[_Bucket, int]]:
        """A free slot of an idle bucket of the job's shape, or a new bucket.  A bucket with a
        chunk in flight admits nothing: its step count and the slots' remaining steps are
        settled when the chunk completes, so the job waits for that (rather than a new bucket)."""
        key = bucket_key(job.config, job.green_kubo)
        busy_room = False
        for b in self.buckets.get(key, []):
            m = b.free_slot()
            if m is not None:
                if b.inflight is None:
                    return b, m
                busy_room = True
        if busy_room:
            return None
        per = self._per_member_bytes(key, job.config)
        if self.budget - self.used < per:
            self._release_idle()
        slots = min(self.max_slots, (self.budget - self.used) // per)
        if slots < 1:
            return None
        b = _Bucket(job.config, int(slots), self.precision, self.seed, self.chunk if self.graphs else 0, job.green_kubo,
                    engine_factory=self.engine_factory, autotune=self.autotune)
        self.used += b.device_bytes
        self.buckets_created += 1
        self.buckets.setdefault(key, []).append(b)
        return b, 0

    def _check_admissible(self, jobs: List[Job]) -> None:
        for job in jobs:
            per = self._per_member_bytes(bucket_key(job.config, job.green_kubo), job.config)
            if per > self.budget:
                raise AdmissionError(f"job {job.key} needs {per} bytes of device memory for one slot, more than the "
                                     f"server's budget of {self.budget} bytes")

    def _finish_chunk(self, b: _Bucket, now: float) -> int:
        n, _ev = b.inflight
        b.inflight = None
        b.engine.synchronize()   # returns at once; raises the engine's device error word (zero density)
        b.step_index += n
        done = 0
        for m, job in enumerate(b.slots):
            if job is None:
                continue
            b.remaining[m] -= n
            if b.remaining[m] == 0:
                job.result = b.engine.get_state(m)
                if b.green_kubo is not None:
                    job.gk_sums, job.gk_blocks = b.engine.gk_read(m, reset=True)
                job.finished = now
                b.engine.set_member(m, key=0, active=False)
                b.slots[m] = None
                done += 1
        return done

    def run(self, jobs: List[Job]) -> Dict[str, float]:
        """Serve `jobs` (arrival times relative to now) until all have finished.

        Each bucket has at most one chunk in flight; chunks of different buckets overlap on the
        device (one stream per engine), and a finished chunk is noticed by polling every event, so
        one slow bucket does not hold back the admissions and launches of the others.  Buckets
        stay with the server between runs (until another shape needs their memory), so a later
        run reuses their engines."""
        self._check_admissible(jobs)
        future = sorted(jobs, key=lambda j: j.arrival)
        pending: List[Job] = []
        t0 = time.perf_counter()
        done = 0
        while done < len(jobs):
            now = time.perf_counter() - t0
            while future and future[0].arrival <= now:
                pending.append(future.pop(0))
            still = []
            for job in pending:
                slot = self._slot_for(job)
                if slot is None:
                    still.append(job)
                else:
                    slot[0].admit(slot[1], job, now)
            pending = still
            inflight = []
            for group in self.buckets.values():
                for b in group:
                    if b.inflight is None and b.active():
                        n = min(self.chunk, min(r for j, r in zip(b.slots, b.remaining) if j is not None))
                        b.engine.step_async(n)
                        b.inflight = (n, self.event_factory(b.engine))
                    if b.inflight is not None:
                        inflight.append(b)
            if not inflight:
                if pending and not future:
                    # every bucket is idle, so _slot_for released them all and still found no room
                    raise AdmissionError(f"{len(pending)} jobs cannot be admitted into an empty server "
                                         f"(budget {self.budget} bytes)")
                if future:
                    time.sleep(max(0.0, min(0.002, future[0].arrival - (time.perf_counter() - t0))))
                continue
            ready = [b for b in inflight if b.inflight[1].query()]
            if not ready:
                # nothing finished yet: poll again shortly (every bucket's event, and the arrivals),
                # so that whichever chunk ends first has its bucket refilled at once
                time.sleep(_POLL_S)
                continue
            now = time.perf_counter() - t0
            for b in ready:
                done += self._finish_chunk(b, now)
        makespan = time.perf_counter() - t0
        lat = np.array([j.latency for j in jobs])
        return {
            "jobs": len(jobs),
            "makespan_s": makespan,
            "steps_per_s": float(sum(j.nsteps for j in jobs) / makespan),
            "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)),
            "buckets": self.buckets_created,
            "buckets_released": self.buckets_released,
        }

    def close(self) -> None:
        for group in self.buckets.values():
            for b in group:
                b.engine.close()
        self.buckets.clear()
        self.used = 0


def job_cost(job: Job) -> float:
    """Relative device work of a job: steps x compute-grid points x fields."""
    c = job.config
    return float(job.nsteps) * c.nx * c.ny * (c.num_order_parameters + 3)


def partition_jobs(jobs: List[Job], world: int) -> List[List[Job]]:
    """Split a stream's jobs over `world` ranks (one server per GPU): longest job first onto
    the least-loaded rank.  Deterministic, so every rank computes the same split."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0.0] * world
    parts: List[List[Job]] = [[] for _ in range(world)]
    for job in sorted(jobs, key=lambda j: (-job_cost(j), j.key)):
        r = min(range(world), key=lambda i: (load[i], i))
        parts[r].append(job)
        load[r] += job_cost(job)
    for p in parts:
        p.sort(key=lambda j: j.arrival)
    return parts


def serve_distributed(server: Server, jobs: List[Job], rank: int, world: int, group=None) -> Dict[str, float]:
    """Serve this rank's share of `jobs` (partition_jobs) and combine the ranks' statistics:
    aggregate steps/s over the slowest rank's makespan, p50/p99 over every job's latency.
    The exchange is one all_gather of (makespan, steps, latencies) after the run, no
    per-step collective."""
    import torch.distributed as dist
    mine = partition_jobs(jobs, world)[rank]
    stats = server.run(mine) if mine else {"makespan_s": 0.0}
    local = {"makespan_s": stats["makespan_s"], "steps": sum(j.nsteps for j in mine), "latency": [j.latency for j in mine],
             "jobs": len(mine)}
    if world > 1:
        gathered: List[dict] = [None] * world  # type: ignore[list-item]
        dist.all_gather_object(gathered, local, group=group)
    else:
        gathered = [local]
    makespan = max(g["makespan_s"] for g in gathered)
    lat = np.array([x for g in gathered for x in g["latency"]])
    return {
        "jobs": sum(g["jobs"] for g in gathered),
        "jobs_per_rank": [g["jobs"] for g in gathered],
        "makespan_s": makespan,
        "steps_per_s": float(sum(g["steps"] for g in gathered) / makespan) if makespan > 0 else 0.0,
        "p50_s": float(np.percentile(lat, 50)),
        "p99_s": float(np.percentile(lat, 99)),
    }


def run_alone(job: Job, precision: int, seed: int) -> np.ndarray:
    """The job on its own (batch of one) with the same noise key and scale as in the server.
    Fills job.gk_sums / gk_blocks when the job asks for the Green-Kubo measure."""
    b = _Bucket(job.config, 1, precision, seed, 0, job.green_kubo)
    b.admit(0, job, 0.0)
    b.engine.step(job.nsteps)
    out = b.engine.get_state(0)
    if b.green_kubo is not None:
        job.gk_sums, job.gk_blocks = b.engine.gk_read(0)
    b.engine.close()
    return out
