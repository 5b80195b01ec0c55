"""The two-pair row pass (kernel family 4: two output pairs per barrier chain, 1 / rho in a
half-line, the (jy, -) line reused as a work line) against the pair-line family and the FP64
oracle, through the C ABI (GPU).

Family 4 applies to compressible dynamics whose last two input pair-lines are (rho, jx),
(jy, -): N = 0, 2, 4 order parameters.  Its products and transforms are the pair-line row
pass's operation for operation, so results agree with family 1 bit for bit.  The cases cover
every pair-line row length (96 ... 1536 points, one to sixteen row pairs per block), an even
and an odd number of output pairs (N = 2: six; N = 0: three; N = 4: nine), the dealiasing
rules, and the zero-density check.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu

TOL32 = 1e-5

CASES = {
    "n2_1536": script(grid=(1024, 1024), length=(2048.0, 2048.0), nop=2, dt=0.01),
    "n2_768x1536": script(grid=(512, 1024), length=(1024.0, 2048.0), nop=2, dt=0.01, eta=0.5, zeta=2.0),
    "n0_384": script(grid=(256, 128), length=(512.0, 256.0), nop=0, dt=0.01, fe=None),
    "n4_192": script(grid=(128, 128), length=(256.0, 256.0), nop=4, dt=0.01),
    "n2_96": script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01),
    "n2_two_768": script(grid=(384, 96), length=(768.0, 192.0), nop=2, dt=0.01, dealias="two"),
}


def _engine(sb, text, family, batch=1):
    cfg = sb.config_from_script(text)
    cfg.precision = sb.FP32
    cfg.batch = batch
    eng = sb.Engine(cfg)
    eng.set_family(family)
    return eng


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_pair_row_pass_rhs(name):
    import shhd_b200 as sb
    text = CASES[name]
    ocfg = so.parse_script(text)
    u = random_state(ocfg, seed=83)
    with _engine(sb, text, 4) as e4:
        assert e4.family == 4
        e4.set_state(u)
        got4 = e4.rhs()
    with _engine(sb, text, 1) as e1:
        assert e1.family == 1
        e1.set_state(u)
        got1 = e1.rhs()
    assert np.array_equal(got4, got1), f"{name}: max |difference| {np.max(np.abs(got4 - got1)):.3e}"
    err = so.rel_l2(got4, so.Oracle(ocfg).rhs(u))
    print(f"{name}: relative L2 against the oracle {err:.3e}")
    assert err < TOL32


@pytest.mark.parametrize("name", ["n2_1536", "n0_384", "n4_192"])
def test_two_pair_row_pass_trajectories(name):
    """Noisy trajectories of two batched members, direct launches and graphs: identical to family 1."""
    import shhd_b200 as sb
    text = CASES[name].replace("run 1", "fix 9 all noise on seed 5 kBT 0.001\nrun 1")
    ocfg = so.parse_script(text)
    us = [random_state(ocfg, seed=95 + m) for m in range(2)]
    out = {}
    for fam, chunk in ((1, 0), (4, 0), (4, 3)):
        with _engine(sb, text, fam, batch=2) as e:
            for m in range(2):
                e.set_state(us[m], member=m)
            if chunk:
                e.set_graph_chunk(chunk)
            e.step(6)
            out[fam, chunk] = [e.get_state(m) for m in range(2)]
    for m in range(2):
        assert np.all(np.isfinite(out[4, 0][m]))
        assert np.array_equal(out[4, 0][m], out[1, 0][m])
        assert np.array_equal(out[4, 3][m], out[1, 0][m])


def test_two_pair_row_pass_scope_and_zero_density():
    import shhd_b200 as sb
    # incompressible and N = 1 layouts have no (rho, jx), (jy, -) lines: family 4 falls back to 1
    for text in (script(grid=(64, 64), length=(128.0, 128.0), nop=1, dt=0.01),
                 script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01, te="srk3/incompressible", cT=None,
                        eta=0.05, zeta=0.0, nonlinear="momentum")):
        with _engine(sb, text, 4) as e:
            assert e.family == 1
    text = script(grid=(1024, 64), length=(2048.0, 128.0), nop=2, dt=0.01)
    with _engine(sb, text, 4) as e:
        assert e.family == 4
        e.set_state(np.zeros(e.shape, complex))
        with pytest.raises(sb.ShhdError) as ei:
            e.step(1)
        assert ei.value.code == sb.SHHD_ENUMERIC and "zero density" in str(ei.value)
