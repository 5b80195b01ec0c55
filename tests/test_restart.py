"""Binary restart files (the reference parses `restart on file` but writes nothing)."""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

TEXT = script(grid=(32, 32), length=(64.0, 64.0), nop=2, dt=0.01, noise="kBT 0.001 seed 3")


def test_restart_round_trip(tmp_path):
    import shhd_b200 as sb
    from shhd_b200 import restart
    cfg = sb.config_from_script(TEXT)
    cfg.batch = 2
    ocfg = so.parse_script(TEXT)
    states = [random_state(ocfg, seed=s) for s in (1, 2)]
    p = tmp_path / "run.restart"
    restart.write_restart(str(p), cfg, states, 123, 1.23)
    c2, s2, step, t = restart.read_restart(str(p))
    assert bytes(memoryview(c2).cast("B")) == bytes(memoryview(cfg).cast("B"))
    assert step == 123 and t == 1.23
    for a, b in zip(states, s2):
        assert np.array_equal(a, b)
    bad = tmp_path / "bad.restart"
    bad.write_bytes(b"NOTARST!" + p.read_bytes()[8:])
    with pytest.raises(ValueError):
        restart.read_restart(str(bad))
    cut = tmp_path / "cut.restart"
    cut.write_bytes(p.read_bytes()[:-16])
    with pytest.raises(ValueError):
        restart.read_restart(str(cut))


@pytest.mark.gpu
def test_resumed_run_continues_the_trajectory(tmp_path):
    """3 steps, save, load into a new engine, 2 steps == 5 uninterrupted steps (noise keyed by step)."""
    import shhd_b200 as sb
    from shhd_b200 import restart
    u0 = random_state(so.parse_script(TEXT), seed=9)
    cfg = sb.config_from_script(TEXT)
    with sb.Engine(cfg) as a, sb.Engine(cfg) as full:
        a.set_state(u0)
        full.set_state(u0)
        a.step(3)
        p = tmp_path / "mid.restart"
        restart.save_engine(str(p), a)
        full.step(3)
        full.step(2)
        with restart.load_engine(str(p)) as b:
            assert b.get_info().step_index == 3
            b.step(2)
            assert so.rel_l2(b.get_state(), full.get_state()) < 1e-15
