"""Continuous-batching server for trajectory jobs (host scheduling over the C ABI).

Jobs of mixed grid, component count and mode arrive over time.  Jobs whose
configurations differ only in temperature and seed share a *bucket*: one
batched engine whose members are slots.  A job is admitted into a free slot
as soon as it has arrived and a slot (or HBM for a new bucket engine) is
free; every scheduling round enqueues one chunk of steps on each bucket with
active slots, each bucket on its own CUDA stream, so buckets overlap on the
device; finished jobs are read back and their slots reused.

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


def _noisy(cfg: Config) -> bool:
    return bool(cfg.noise_momentum or cfg.noise_order_parameter)


class _Bucket:
    def __init__(self, cfg: Config, slots: int, precision: int, seed: int, graph_chunk: int = 0,
                 green_kubo: Optional[Tuple[int, int]] = None):
        c = cfg.copy()
        c.batch = slots
        c.precision = precision
        c.noise_seed = seed
        c.member_offset = 0
        if _noisy(cfg):
            c.kBT = 1.0  # members carry sqrt(kBT_job) as their amplitude factor
        self.engine = Engine(c)
        if graph_chunk > 0:
            self.engine.set_graph_chunk(graph_chunk)
        self.green_kubo = green_kubo
        if green_kubo is not None:
            self.engine.gk_enable(*green_kubo)
        self.slots: List[Optional[Job]] = [None] * slots
        self.remaining = [0] * slots
        self.step_index = 0
        self.noisy = _noisy(cfg)
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
        self.slots[m] = job
        self.remaining[m] = job.nsteps
        job.admitted = now

    def active(self) -> bool:
        return any(j is not None for j in self.slots)


class Server:
    def __init__(self, precision: int = FP32, seed: int = 20240601, max_slots: int = 32, chunk: int = 25,
                 hbm_budget: Optional[int] = None, graphs: bool = True):
        import torch
        self.graphs = graphs
        self.precision = precision
        self.seed = seed
        self.max_slots = max_slots
        self.chunk = chunk
        free, _total = torch.cuda.mem_get_info()
        self.budget = int(0.8 * free) if hbm_budget is None else int(hbm_budget)
        self.used = 0
        self.buckets: Dict[bytes, List[_Bucket]] = {}
        self._member_bytes: Dict[bytes, int] = {}

    def _per_member_bytes(self, key: bytes, cfg: Config) -> int:
        if key not in self._member_bytes:
            c = cfg.copy()
            c.batch = 1
            c.precision = self.precision
            with Engine(c) as probe:
                self._member_bytes[key] = int(probe.get_info().device_bytes) + probe.info.state_doubles * 8
        return self._member_bytes[key]

    def _slot_for(self, job: Job) -> Optional[Tuple[_Bucket, int]]:
        key = bucket_key(job.config, job.green_kubo)
        for b in self.buckets.get(key, []):
            m = b.free_slot()
            if m is not None:
                return b, m
        per = self._per_member_bytes(key, job.config)
        slots = min(self.max_slots, (self.budget - self.used) // per)
        if slots < 1:
            return None
        b = _Bucket(job.config, int(slots), self.precision, self.seed, self.chunk if self.graphs else 0, job.green_kubo)
        self.used += int(b.engine.get_info().device_bytes)
        self.buckets.setdefault(key, []).append(b)
        return b, 0

    def run(self, jobs: List[Job]) -> Dict[str, float]:
        """Serve `jobs` (arrival times relative to now) until all have finished."""
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
            stepped = []
            for group in self.buckets.values():
                for b in group:
                    if not b.active():
                        continue
                    n = min(self.chunk, min(r for j, r in zip(b.slots, b.remaining) if j is not None))
                    b.engine.step_async(n)
                    stepped.append((b, n))
            if not stepped:
                if future:
                    time.sleep(max(0.0, min(0.002, future[0].arrival - (time.perf_counter() - t0))))
                continue
            for b, n in stepped:
                b.engine.synchronize()
                b.step_index += n
                now = time.perf_counter() - t0
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
        makespan = time.perf_counter() - t0
        lat = np.array([j.latency for j in jobs])
        return {
            "jobs": len(jobs),
            "makespan_s": makespan,
            "steps_per_s": float(sum(j.nsteps for j in jobs) / makespan),
            "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)),
            "buckets": sum(len(v) for v in self.buckets.values()),
        }

    def close(self) -> None:
        for group in self.buckets.values():
            for b in group:
                b.engine.close()
        self.buckets.clear()


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
