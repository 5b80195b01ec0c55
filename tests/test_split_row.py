"""The split row pass (kernel family 3: x-inverse kernel, physical-row buffer, forward kernel per
output pair) against the FP64 oracle and against the pair-line family, through the C ABI (GPU).

It applies to every FP32 pair-line size (compute rows of 96 ... 1536 points); the cases cover
several row pairs per block (96, 384, 768 points) and one (1536), compressible with the
canonical line layout (1 / rho stored for the velocity) and without it, incompressible
(v = j / rho0), quiescent, and the dealiasing rules.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu

TOL32 = 1e-5

CASES = {
    "comp_n2_1536": script(grid=(1024, 1024), length=(2048.0, 2048.0), nop=2, dt=0.01),
    "comp_n1_1536x768": script(grid=(1024, 512), length=(2048.0, 1024.0), nop=1, dt=0.01, eta=0.5, zeta=2.0),
    "incomp_n0_768": script(grid=(512, 256), length=(1024.0, 512.0), nop=0, dt=0.01, te="srk3/incompressible", cT=None, eta=0.05,
                            zeta=0.0, nonlinear="momentum"),
    "quiescent_n1_384": script(grid=(256, 256), length=(512.0, 512.0), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0,
                               zeta=0.0, nonlinear=None),
    "comp_n3_96": script(grid=(64, 64), length=(128.0, 128.0), nop=3, dt=0.01),
    "comp_n2_two_768": script(grid=(384, 96), length=(768.0, 192.0), nop=2, dt=0.01, dealias="two"),
}


def _engine(sb, text, family, batch=1):
    cfg = sb.config_from_script(text)
    cfg.precision = sb.FP32
    cfg.batch = batch
    eng = sb.Engine(cfg)
    eng.set_family(family)
    return eng


@pytest.mark.parametrize("name", sorted(CASES))
def test_split_row_pass_rhs_matches_oracle(name):
    import shhd_b200 as sb
    text = CASES[name]
    ocfg = so.parse_script(text)
    u = random_state(ocfg, seed=81, transverse=ocfg.mode == "incompressible")
    want = so.Oracle(ocfg).rhs(u)
    with _engine(sb, text, 3) as e3:
        assert e3.family == 3
        e3.set_state(u)
        got3 = e3.rhs()
    with _engine(sb, text, 1) as e1:
        e1.set_state(u)
        got1 = e1.rhs()
    err3, err1 = so.rel_l2(got3, want), so.rel_l2(got1, want)
    print(f"{name}: relative L2 against the oracle: split row pass {err3:.3e}, pair-line {err1:.3e}")
    assert err3 < TOL32


@pytest.mark.parametrize("name", ["comp_n2_1536", "incomp_n0_768", "quiescent_n1_384"])
def test_split_row_pass_trajectory_and_members(name):
    """Noisy trajectories of two batched members under family 3 equal family 1's within FP32
    round-off (same Philox noise)."""
    import shhd_b200 as sb
    text = CASES[name].replace("run 1", "fix 9 all noise on seed 5 kBT 0.001\nrun 1")
    ocfg = so.parse_script(text)
    us = [random_state(ocfg, seed=90 + m, transverse=ocfg.mode == "incompressible") for m in range(2)]
    out = {}
    for fam in (1, 3):
        with _engine(sb, text, fam, batch=2) as e:
            for m in range(2):
                e.set_state(us[m], member=m)
            e.step(6)
            out[fam] = [e.get_state(m) for m in range(2)]
    for m in range(2):
        assert np.all(np.isfinite(out[3][m]))
        assert so.rel_l2(out[3][m], out[1][m]) < TOL32


def test_split_row_pass_zero_density_graphs_and_family_switch():
    import shhd_b200 as sb
    text = script(grid=(1024, 64), length=(2048.0, 128.0), nop=0, dt=0.01)
    ocfg = so.parse_script(text)
    with _engine(sb, text, 3) as e:
        e.set_state(np.zeros(e.shape, complex))
        with pytest.raises(sb.ShhdError) as ei:
            e.step(1)
        assert ei.value.code == sb.SHHD_ENUMERIC and "zero density" in str(ei.value)
    u = random_state(ocfg, seed=3)
    text_n = text.replace("run 1", "fix 9 all noise on seed 2 kBT 0.001\nrun 1")
    res = []
    for chunk in (0, 4):
        with _engine(sb, text_n, 3) as e:
            e.set_state(u)
            if chunk:
                e.set_graph_chunk(chunk)
            e.step(8)
            res.append(e.get_state())
    assert np.array_equal(res[0], res[1])
    # leaving the family frees its buffer; coming back allocates it again
    with _engine(sb, text_n, 3) as e:
        b3 = e.get_info().device_bytes
        e.set_family(1)
        assert e.get_info().device_bytes < b3
        e.set_family(3)
        assert e.get_info().device_bytes == b3
        e.set_state(u)
        e.step(2)
        assert np.all(np.isfinite(e.get_state()))


@pytest.mark.parametrize("grid", [(64, 64), (256, 128), (512, 512)])
def test_packed_row_pairs_match_unpacked(grid):
    """One input slot and one output (quiescent, N = 1): the pair-line row pass packs two row
    pairs into one pair-line; its results equal the split row pass's, which transforms the same
    lines unpacked, bit for bit (each half's arithmetic is the same operations)."""
    import shhd_b200 as sb
    text = script(grid=grid, length=(2.0 * grid[0], 2.0 * grid[1]), nop=1, dt=0.02, te="srk3/quiescent", cT=None, eta=0.0,
                  zeta=0.0, nonlinear=None).replace("run 1", "fix 9 all noise on seed 3 kBT 0.01\nrun 1")
    ocfg = so.parse_script(text)
    u = random_state(ocfg, seed=17, amp=0.3)
    out = {}
    for fam in (1, 3):
        with _engine(sb, text, fam, batch=2) as e:
            for m in range(2):
                e.set_state(u, member=m)
            out[fam, "rhs"] = e.rhs()
            e.step(4)
            out[fam, "state"] = e.get_state(1)
    assert np.array_equal(out[1, "rhs"], out[3, "rhs"])
    assert np.array_equal(out[1, "state"], out[3, "state"])
    assert so.rel_l2(out[1, "rhs"], so.Oracle(ocfg).rhs(u)) < TOL32
