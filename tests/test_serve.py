"""Serving loop: continuous batching of mixed jobs; each result equals the job run alone (GPU)."""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu


def _jobs(sb, serve):
    specs = [
        (script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, noise="kBT 0.002 seed 1"), 40, 0.000),
        (script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, noise="kBT 0.0005 seed 9"), 65, 0.005),
        (script(grid=(128, 128), length=(256.0, 256.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0, zeta=0.0,
                nonlinear=None, noise="kBT 0.01 seed 2"), 30, 0.010),
        (script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, noise="kBT 0.004 seed 3"), 25, 0.020),
        (script(grid=(128, 128), length=(256.0, 256.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0, zeta=0.0,
                nonlinear=None, noise="kBT 0.03 seed 4"), 55, 0.030),
        (script(grid=(64, 64), length=(128.0, 128.0), nop=0, dt=0.01, te="srk3/incompressible", cT=None, eta=0.05, zeta=0.0,
                nonlinear="momentum", noise="kBT 0.001 seed 5"), 35, 0.040),
    ]
    jobs = []
    for k, (text, n, t) in enumerate(specs):
        cfg = sb.config_from_script(text)
        ocfg = so.parse_script(text)
        st = random_state(ocfg, seed=100 + k, amp=0.03, transverse=(ocfg.mode == "incompressible"))
        jobs.append(serve.Job(key=1000 + k, config=cfg, state=st, nsteps=n, arrival=t))
    return jobs


@pytest.mark.parametrize("precision", [0, 1])
def test_served_results_equal_alone(precision):
    import shhd_b200 as sb
    from shhd_b200 import serve
    jobs = _jobs(sb, serve)
    srv = serve.Server(precision=precision, seed=77, max_slots=4, chunk=10)
    stats = srv.run(jobs)
    srv.close()
    assert stats["jobs"] == len(jobs)
    assert stats["p50_s"] <= stats["p99_s"]
    assert stats["buckets"] >= 3  # three distinct configurations
    for job in jobs:
        alone = serve.run_alone(job, precision, seed=77)
        assert job.result is not None
        assert so.rel_l2(job.result, alone) < 1e-13, job.key


def test_inactive_members_are_untouched():
    import shhd_b200 as sb
    text = script(grid=(64, 64), length=(128.0, 128.0), nop=1, dt=0.01, noise="kBT 0.002 seed 1")
    cfg = sb.config_from_script(text)
    cfg.batch = 2
    ocfg = so.parse_script(text)
    a, b = random_state(ocfg, seed=1), random_state(ocfg, seed=2)
    with sb.Engine(cfg) as eng:
        eng.set_state(a, member=0)
        eng.set_state(b, member=1)
        eng.set_member(1, key=5, active=False)
        eng.step(3)
        assert np.array_equal(eng.get_state(1), b)
        assert not np.array_equal(eng.get_state(0), a)


def test_engines_sharing_a_kernel_size_coexist():
    """Two engines of one compute size but different shared-memory needs (5 and 2 transformed
    fields at 96^2): creating the smaller one must not break launches of the larger one."""
    import shhd_b200 as sb
    big = script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01)
    small = script(grid=(64, 64), length=(128.0, 128.0), nop=0, dt=0.01, te="srk3/incompressible", cT=None, eta=0.05,
                   zeta=0.0, nonlinear="momentum")
    ob, osm = so.parse_script(big), so.parse_script(small)
    ub, us = random_state(ob, seed=3), random_state(osm, seed=4, transverse=True)
    with sb.Engine(sb.config_from_script(big)) as eb, sb.Engine(sb.config_from_script(small)) as es:
        eb.set_state(ub)
        es.set_state(us)
        eb.step(2)
        es.step(2)
        ref = so.Oracle(ob)
        u = ub
        for _ in range(2):
            u = ref.step(u, "philox")
        assert so.rel_l2(eb.get_state(), u) < 1e-12


def test_served_green_kubo_equals_alone():
    """Green-Kubo sums of a served job (slots reused, other jobs running) equal the job run alone."""
    import shhd_b200 as sb
    from shhd_b200 import serve
    text = script(grid=(32, 32), length=(64.0, 64.0), nop=1, dt=0.01, eta=0.5, zeta=0.5, noise="kBT 0.002 seed 1")
    ocfg = so.parse_script(text)
    jobs = [serve.Job(key=500 + k, config=sb.config_from_script(text), state=random_state(ocfg, seed=60 + k), nsteps=n,
                      arrival=0.002 * k, green_kubo=(2, 8)) for k, n in enumerate((24, 40, 16, 32))]
    srv = serve.Server(precision=0, seed=5, max_slots=2, chunk=8)
    srv.run(jobs)
    srv.close()
    for job in jobs:
        sums, blocks = job.gk_sums, job.gk_blocks
        alone = serve.Job(key=job.key, config=job.config, state=job.state, nsteps=job.nsteps, green_kubo=(2, 8))
        serve.run_alone(alone, 0, seed=5)
        assert blocks == alone.gk_blocks == job.nsteps // 8
        assert np.abs(sums - alone.gk_sums).max() <= 1e-12 * np.abs(alone.gk_sums).max()


def test_jobs_from_set_lines_equal_jobs_with_host_states():
    """A job may carry its `set` lines instead of a state: admission generates it on the device."""
    import shhd_b200 as sb
    from shhd_b200 import serve
    from shhd_b200.initial import initial_state
    base = script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, noise="kBT 0.002 seed 1")
    jobs_dev, jobs_host = [], []
    for k in range(3):
        text = base + "\n".join([
            "",
            f"set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed {10 + k}",
            f"set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed {20 + k}",
            f"set order_parameter all equilibrium/gaussian seed {30 + k} kBT 0.002 k0 2 k2 1",
        ])
        cfg = sb.config_from_script(text)
        jobs_dev.append(serve.Job(key=500 + k, config=cfg, state=None, initial=text, nsteps=20 + 5 * k, arrival=0.002 * k))
        jobs_host.append(serve.Job(key=500 + k, config=cfg, state=initial_state(cfg, text), nsteps=20 + 5 * k,
                                   arrival=0.002 * k))
    for jobs in (jobs_dev, jobs_host):
        srv = serve.Server(precision=0, seed=5, max_slots=2, chunk=5)
        srv.run(jobs)
        srv.close()
    for a, b in zip(jobs_dev, jobs_host):
        assert np.all(np.isfinite(a.result))
        assert so.rel_l2(a.result, b.result) < 1e-12, a.key
