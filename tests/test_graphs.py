"""Captured CUDA graph replay of step chunks (GPU).

A replayed chunk must reproduce the direct launches exactly: the captured
kernels are the same launches, and the noise is keyed by the device-side step
counter that each replay advances.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu

# grid spacing 2: the phi4 gradient term -M k^2 (a + b k^2) stays inside the
# integrators' stability intervals at these time steps for every active mode
SRK3 = script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, noise="kBT 0.001 seed 3")
EULER = script(grid=(48, 32), length=(96.0, 64.0), nop=1, dt=0.005, te="euler/compressible", eta=0.5, zeta=2.0,
               noise="kBT 0.002 seed 4")
QUIET = script(grid=(128, 128), length=(256.0, 256.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0, zeta=0.0,
               nonlinear=None, noise="kBT 0.05 seed 5")


def _engine(sb, text, precision, batch=1):
    cfg = sb.config_from_script(text)
    cfg.precision = precision
    cfg.batch = batch
    return sb.Engine(cfg)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,text", [("srk3", SRK3), ("quiescent", QUIET)])
def test_graph_replay_equals_direct_launches(precision, name, text):
    import shhd_b200 as sb
    u0 = random_state(so.parse_script(text), seed=11)
    with _engine(sb, text, precision, batch=2) as g, _engine(sb, text, precision, batch=2) as d:
        for m in range(2):
            g.set_state(u0, member=m)
            d.set_state(u0, member=m)
        g.set_graph_chunk(3)
        g.step(7)          # two replays of 3 steps, then one direct step
        g.step(3)          # one more replay
        for n in (3, 3, 1, 3):
            d.step(n)
        for m in range(2):
            got = g.get_state(m)
            assert np.all(np.isfinite(got))
            assert np.array_equal(got, d.get_state(m)), (name, precision, m)
        assert g.get_info().step_index == d.get_info().step_index == 10
        # launches are counted for replays as for direct calls
        sg, sd = g.kernel_stats(), d.kernel_stats()
        for k in ("col_inverse", "row_pass", "col_forward"):
            assert sg[k][1] == sd[k][1], k


def test_graph_replay_matches_the_oracle():
    import shhd_b200 as sb
    cfg = so.parse_script(SRK3)
    u0 = random_state(cfg, seed=2)
    o = so.Oracle(cfg)
    ref = u0
    for _ in range(6):
        ref = o.step(ref, "philox")
    with _engine(sb, SRK3, 0) as g:
        g.set_state(u0)
        g.set_graph_chunk(2)
        g.step(6)
        assert so.rel_l2(g.get_state(), ref) < 1e-12


def test_euler_chunks_round_to_even():
    import shhd_b200 as sb
    u0 = random_state(so.parse_script(EULER), seed=5)
    with _engine(sb, EULER, 0) as g, _engine(sb, EULER, 0) as d:
        g.set_state(u0)
        d.set_state(u0)
        g.set_graph_chunk(3)   # Euler swaps its buffers each step: rounded up to 4
        g.step(8)
        d.step(4)
        d.step(4)
        got = g.get_state()
        assert np.all(np.isfinite(got))
        assert np.array_equal(got, d.get_state())


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_restores_state_and_keeps_results(precision):
    import shhd_b200 as sb
    cfg = so.parse_script(SRK3)
    u0 = random_state(cfg, seed=21)
    ref = u0
    o = so.Oracle(cfg)
    for _ in range(4):
        ref = o.step(ref, "philox")
    with _engine(sb, SRK3, precision) as e:
        e.set_state(u0)
        before = e.get_state()
        choice = e.autotune(2)
        # FP32 at a 96-point compute grid: single-line, pair-line, split and two-pair row passes,
        # each direct and through graphs (the register row pass exists for 1536-point rows only)
        fp32_families = ("pair-line", "single-line", "pair-line + split row pass", "pair-line + two-pair row pass")
        assert choice["family"] in (fp32_families if precision == 1 else ("single-line",))
        timed = [x for x in choice["ms_per_step"] if x is not None]
        assert len(timed) == (8 if precision == 1 else 2) and all(x > 0 for x in timed)
        assert e.get_info().step_index == 0
        assert np.array_equal(e.get_state(), before)
        e.step(4)
        assert so.rel_l2(e.get_state(), ref) < (1e-12 if precision == 0 else 1e-5)


SHAPES = {
    # 384-point rows and columns, one input pair-line, no momentum group: both kernels have a choice
    "quiescent_384": script(grid=(256, 256), length=(512.0, 512.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None,
                            eta=0.0, zeta=0.0, nonlinear=None, noise="kBT 0.05 seed 5"),
    # 768-point rows and columns, compressible N = 2 (three input pair-lines, a momentum group)
    "compressible_768": script(grid=(512, 512), length=(1024.0, 1024.0), nop=2, dt=0.01, noise="kBT 0.001 seed 3"),
}


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_launch_shapes_give_identical_results(name):
    """Every launch shape of the pair-line kernels runs the same code at another register budget:
    the RHS and a noisy trajectory agree bit for bit with the rule's shape."""
    import shhd_b200 as sb
    text = SHAPES[name]
    u0 = random_state(so.parse_script(text), seed=31)
    out = {}
    for shape in ((0, 0), (2, 3), (2, 4), (3, 3), (3, 4)):
        with _engine(sb, text, sb.FP32) as e:
            assert e.family == 1
            e.set_launch_shape(*shape)
            row, col = e.launch_shape
            if shape != (0, 0):
                assert (row, col) == shape
            e.set_state(u0)
            rhs = e.rhs()
            e.step(4)
            out[shape] = (rhs, e.get_state())
    for shape, (rhs, state) in out.items():
        assert np.all(np.isfinite(state))
        assert np.array_equal(rhs, out[0, 0][0]), (name, shape)
        assert np.array_equal(state, out[0, 0][1]), (name, shape)


def test_launch_shape_rules_and_autotune():
    import shhd_b200 as sb
    with _engine(sb, SHAPES["quiescent_384"], sb.FP32) as e:
        assert e.launch_shape == (3, 4)          # 1 input pair-line, no momentum group: both at the higher count
        with pytest.raises(sb.ShhdError) as ei:
            e.set_launch_shape(4, 0)
        assert ei.value.code == sb.SHHD_EINVAL
        with pytest.raises(sb.ShhdError):
            e.set_launch_shape(0, 2)
        e.set_state(random_state(so.parse_script(SHAPES["quiescent_384"]), seed=32))
        choice = e.autotune(2)
        assert e.launch_shape == (choice["launch_shape"]["row_blocks"], choice["launch_shape"]["col_blocks"])
        if choice["family"] == "pair-line":
            assert e.launch_shape[0] in (2, 3) and e.launch_shape[1] in (3, 4)
    with _engine(sb, SHAPES["compressible_768"], sb.FP32) as e:
        assert e.launch_shape[1] == 3            # momentum group on 768-point columns: three
    with _engine(sb, SRK3, sb.FP64) as e:
        assert e.launch_shape == (0, 0)          # no pair-line kernels


def test_batch_above_the_grid_limit_is_refused():
    """Members are a grid dimension of the stage kernels: more than 65535 is refused at creation."""
    import shhd_b200 as sb
    cfg = sb.config_from_script(SRK3)
    cfg.batch = 65536
    with pytest.raises(sb.ShhdError) as ei:
        sb.Engine(cfg)
    assert ei.value.code == sb.SHHD_EINVAL and "batch must be <= 65535" in str(ei.value)
