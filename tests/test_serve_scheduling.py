"""Scheduling of the serving loop without a GPU: budget exhaustion, release of idle buckets,
refusal of jobs no empty server can hold, partition over ranks (gloo, world size 2).

A fake engine stands in for the device: it counts steps and reports a device size
proportional to its slots, so the admission and release logic runs as on a GPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from helpers import script


class FakeInfo:
    def __init__(self, device_bytes, state_doubles):
        self.device_bytes = device_bytes
        self.state_doubles = state_doubles


class FakeEvent:
    def __init__(self, polls=1):
        self.polls = polls

    def query(self):
        self.polls -= 1
        return self.polls < 0

    def synchronize(self):
        self.polls = -1


class FakeEngine:
    """Device size = 1000 bytes per slot per compute-grid point unit; steps are counted per member."""
    live = []

    def __init__(self, cfg):
        self.cfg = cfg.copy()
        self.batch = cfg.batch
        self.unit = cfg.nx * cfg.ny // 1024
        self.info = FakeInfo(1000 * self.unit * self.batch, 10)
        self.steps = np.zeros(self.batch, dtype=int)
        self.active = np.zeros(self.batch, dtype=bool)
        self.closed = False
        self.stream = 0
        FakeEngine.live.append(self)

    def get_info(self):
        return self.info

    def set_graph_chunk(self, n):
        self.chunks = getattr(self, "chunks", []) + [n]

    def autotune(self, trial_steps):
        # the real engine restores state and step count; here: record the call and what was active
        self.tuned = getattr(self, "tuned", []) + [(trial_steps, int(self.active.sum()))]

    def gk_enable(self, *a):
        pass

    def set_member(self, m, key, step_origin=0, noise_scale=1.0, active=True):
        self.active[m] = active
        if active:
            self.steps[m] = 0

    def set_state(self, state, member=0):
        pass

    def get_state(self, member=0):
        return np.array([self.steps[member]])

    def step_async(self, n):
        assert not self.closed
        self.steps[self.active] += n

    def synchronize(self):
        pass

    def close(self):
        self.closed = True


def _cfg(grid):
    import shhd_b200 as sb
    return sb.config_from_script(script(grid=(grid, grid), length=(2.0 * grid, 2.0 * grid), nop=1, dt=0.01))


def _server(budget, **kw):
    from shhd_b200 import serve
    return serve.Server(precision=1, seed=1, hbm_budget=budget, engine_factory=FakeEngine,
                        event_factory=lambda eng: FakeEvent(1), **kw)


def test_shapes_exceeding_the_budget_run_in_sequence():
    """Each shape's bucket fits alone but no two fit together: idle buckets are released and
    every job finishes with exactly its own step count."""
    from shhd_b200 import serve
    FakeEngine.live = []
    # compute grids 96^2 (9 units/slot), 192^2 (36), 384^2 (144); budget 150 units: one bucket of one slot at a time
    # for the large shape, several small slots otherwise
    jobs = []
    for k, (g, n) in enumerate([(64, 30), (128, 20), (256, 40), (64, 10), (256, 15), (128, 25)]):
        jobs.append(serve.Job(key=k, config=_cfg(g), state=None, initial="set density uniform value 1.0", nsteps=n, arrival=0.0))
    for j in jobs:
        j.state = np.zeros(1)
    srv = _server(150 * 1000, max_slots=2, chunk=7)
    stats = srv.run(jobs)
    assert stats["jobs"] == len(jobs)
    for j in jobs:
        assert int(j.result[0]) == j.nsteps, (j.key, j.result, j.nsteps)
    assert stats["buckets_released"] >= 1
    assert 0 <= srv.used <= srv.budget
    srv.close()
    assert all(e.closed for e in FakeEngine.live)


def test_job_larger_than_an_empty_server_is_refused():
    from shhd_b200 import serve
    FakeEngine.live = []
    big = serve.Job(key=1, config=_cfg(256), state=np.zeros(1), nsteps=5)
    small = serve.Job(key=2, config=_cfg(64), state=np.zeros(1), nsteps=5)
    srv = _server(50 * 1000)
    with pytest.raises(serve.AdmissionError, match="more than the server's budget"):
        srv.run([small, big])
    assert small.result is None  # refused before anything ran
    srv.close()


def test_partition_covers_every_job_once_and_balances():
    from shhd_b200 import serve
    rng = np.random.default_rng(0)
    jobs = [serve.Job(key=k, config=_cfg(int(rng.choice([64, 128, 256]))), state=None, nsteps=int(rng.integers(10, 100)),
                      arrival=float(k)) for k in range(40)]
    for world in (1, 2, 3, 8):
        parts = serve.partition_jobs(jobs, world)
        keys = sorted(j.key for p in parts for j in p)
        assert keys == list(range(40))
        loads = [sum(serve.job_cost(j) for j in p) for p in parts]
        assert max(loads) - min(loads) <= max(serve.job_cost(j) for j in jobs)
        for p in parts:
            assert [j.arrival for j in p] == sorted(j.arrival for j in p)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dist_worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from shhd_b200 import serve
        jobs = [serve.Job(key=k, config=_cfg((64, 128)[k % 2]), state=np.zeros(1), nsteps=10 + 5 * k, arrival=0.0)
                for k in range(7)]
        srv = _server(10 ** 9, max_slots=4, chunk=6)
        stats = serve.serve_distributed(srv, jobs, rank, world)
        mine = serve.partition_jobs(jobs, world)[rank]
        ok = all(int(j.result[0]) == j.nsteps for j in mine)
        out[rank] = (stats["jobs"], stats["jobs_per_rank"], ok, sorted(j.key for j in mine))
        srv.close()
    finally:
        dist.destroy_process_group()


def test_served_stream_partitioned_over_two_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_dist_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
            assert p.exitcode == 0
        assert out[0][0] == out[1][0] == 7
        assert out[0][1] == out[1][1] and sum(out[0][1]) == 7
        assert out[0][2] and out[1][2]
        assert sorted(out[0][3] + out[1][3]) == list(range(7))


def test_jobs_arriving_while_chunks_are_in_flight():
    """Arrivals land while their bucket's chunk is in flight (two shapes, so while the oldest chunk
    is waited for the other bucket's stays in flight; slow events): each job still takes exactly
    its own step count, counted from its own admission."""
    from shhd_b200 import serve
    FakeEngine.live = []
    jobs = [serve.Job(key=k, config=_cfg((64, 128)[k % 2]), state=np.zeros(1), nsteps=60 + 7 * k, arrival=0.00002 * k)
            for k in range(12)]
    srv = serve.Server(precision=1, seed=1, hbm_budget=10 ** 9, max_slots=4, chunk=5, engine_factory=FakeEngine,
                       event_factory=lambda eng: FakeEvent(40))
    stats = srv.run(jobs)
    assert stats["jobs"] == 12
    for j in jobs:
        assert int(j.result[0]) == j.nsteps, (j.key, int(j.result[0]), j.nsteps)
    srv.close()


def test_each_new_bucket_autotunes_once_on_its_first_job():
    from shhd_b200 import serve
    FakeEngine.live = []
    jobs = [serve.Job(key=k, config=_cfg(g), state=np.zeros(1), nsteps=n, arrival=0.0)
            for k, (g, n) in enumerate([(64, 30), (128, 20), (64, 10), (128, 25), (64, 5)])]
    srv = _server(10 ** 9, max_slots=4, chunk=7, autotune=3)
    srv.run(jobs)
    engines = [e for e in FakeEngine.live if e.batch > 1 or getattr(e, "chunks", None)]
    assert len(engines) == 2
    for e in engines:
        assert e.tuned == [(3, 1)]          # once, with the first job's slot active
        assert e.chunks == [7, 7]           # the server's chunk set again after the autotuner's choice
    for j in jobs:
        assert int(j.result[0]) == j.nsteps
    srv.close()
