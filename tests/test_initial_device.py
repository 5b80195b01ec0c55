"""Initial conditions generated on the device (shhd_engine_set_gaussian_field).

The CPU test evaluates the per-field generators with numpy and checks them
against the reference's own initial states (golden u0), so the mapping of
`set` lines to (seed, channel, mean, s0, c0, c2, c4) is pinned without a GPU.
The GPU tests check the kernel's draws against the same states: FP64 engines
to 1e-13 relative L2 (the device's log/sin/cos differ from numpy's by an ulp
or two), FP32 engines to 1e-6 (one rounding to float per component) with the
k = 0 modes exact, because FP32 engines keep those in FP64.
"""
import math

import numpy as np
import pytest

import shhd_oracle as so
from helpers import load_golden, script

CASES = load_golden()
SUPPORTED = ("uniform", "equilibrium/gaussian", "equilibrium/gaussian/compressible")


def _supported(text):
    for line in text.splitlines():
        t = line.split()
        if t and t[0] == "set":
            style = t[2] if t[1] in ("density", "rho") else t[3]
            if style not in SUPPORTED:
                return False
    return True


NAMES = sorted(n for n, c in CASES.items() if _supported(c["script"]))


def _evaluate(cfg, gens):
    """The state the generators describe, on the host (numpy restatement of the device kernel)."""
    from shhd_b200.initial import _Grid
    g = _Grid((cfg.active_nx, cfg.active_ny), (cfg.nx, cfg.ny), (cfg.lx, cfg.ly))
    u = np.zeros((len(gens), g.ny, g.hx), dtype=np.complex128)
    use = g.active & (g.k2 != 0.0)
    for f, seed, channel, mean, s0, c0, c2, c4 in gens:
        if s0 != 0.0:
            with np.errstate(divide="ignore", invalid="ignore"):
                sigma = np.sqrt(s0 / (c0 + c2 * g.k2 + c4 * g.k2 * g.k2))
            u[f] = np.where(use, sigma * g.gaussian_modes(seed, channel), 0.0)
        u[f, 0, 0] = mean
    return u


@pytest.mark.parametrize("name", NAMES)
def test_generators_reproduce_reference_states(name):
    import shhd_b200 as sb
    from shhd_b200.initial import field_generators
    c = CASES[name]
    cfg = sb.config_from_script(c["script"])
    u = _evaluate(cfg, field_generators(cfg, c["script"]))
    assert so.rel_l2(u, c["u0"]) < 1e-14


def test_generators_last_command_wins_and_missing_fields_are_zero():
    import shhd_b200 as sb
    from shhd_b200.initial import field_generators, initial_state
    text = script(grid=(32, 32), nop=2) + "\n".join([
        "",
        "set density uniform value 2.0",
        "set density equilibrium/gaussian kBT 1e-3 rho0 1.5 cT 1 seed 3",
        "set order_parameter 1 equilibrium/gaussian seed 2 kBT 1 k0 4 k2 1",
        "set order_parameter 1 uniform value 0.25",
        "set momentum x equilibrium/gaussian/compressible kBT 1e-3 seed 6",
    ])
    cfg = sb.config_from_script(text)
    gens = field_generators(cfg, text)
    assert so.rel_l2(_evaluate(cfg, gens), initial_state(cfg, text)) < 1e-14
    ng = cfg.nx * cfg.ny                            # the 3/2-padded transform grid, 48 x 48
    cell = cfg.lx * cfg.ly / ng
    assert gens[1][3:5] == (0.0, 0.0)              # order parameter 0: never set
    assert gens[2][3:5] == (0.25 * ng, 0.0)        # order parameter 1: the uniform command came last
    assert gens[4][4] == 0.0                       # momentum y: never set
    assert math.isclose(gens[3][4], 1e-3 * ng * 1.5 / (2.0 * cell))  # momentum x reads rho0 = 1.5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", NAMES)
def test_device_initial_state_matches_host(name, precision):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    c = CASES[name]
    cfg = sb.config_from_script(c["script"])
    cfg.precision = precision
    cfg.batch = 2
    with sb.Engine(cfg) as eng:
        other = np.full_like(c["u0"], 0.0)
        eng.set_state(c["u0"] * 0.5, member=0)   # the generated member is overwritten everywhere
        eng.set_state(other, member=1)
        initial_state_device(eng, c["script"], member=0)
        got = eng.get_state(0)
        tol = 1e-13 if precision == 0 else 1e-6
        assert so.rel_l2(got, c["u0"]) < tol
        assert np.array_equal(got[:, 0, 0], c["u0"][:, 0, 0])
        assert np.array_equal(eng.get_state(1), other)


@pytest.mark.gpu
def test_device_initial_state_steps_like_the_uploaded_state():
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    c = CASES["srk3_compressible_n2"]
    cfg = sb.config_from_script(c["script"])
    with sb.Engine(cfg) as a, sb.Engine(cfg) as b:
        initial_state_device(a, c["script"])
        b.set_state(c["u0"])
        a.step(3)
        b.step(3)
        assert so.rel_l2(a.get_state(), b.get_state()) < 1e-12


@pytest.mark.gpu
def test_device_initial_state_full_size():
    """1024^2 grid (1536^2 transforms), two order parameters: the benchmark-size initial state."""
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state, initial_state_device
    text = script(grid=(1024, 1024), length=(2048.0, 2048.0), nop=2, dt=0.01) + "\n".join([
        "",
        "set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 11",
        "set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 12",
        "set order_parameter all equilibrium/gaussian seed 13 kBT 0.04 k0 2 k2 1",
    ])
    cfg = sb.config_from_script(text)
    with sb.Engine(cfg) as eng:
        initial_state_device(eng, text)
        assert so.rel_l2(eng.get_state(), initial_state(cfg, text)) < 1e-13


@pytest.mark.gpu
def test_device_initial_state_rejects_a_nonpositive_coefficient():
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    text = script(grid=(32, 32), nop=1) + "\nset order_parameter all equilibrium/gaussian seed 1 kBT 1 k0 -1 k2 0\n"
    cfg = sb.config_from_script(text)
    with sb.Engine(cfg) as eng:
        with pytest.raises(sb.ShhdError) as ei:
            initial_state_device(eng, text)
        assert ei.value.code == sb.SHHD_EINVAL
        assert "positive linear chemical-potential" in str(ei.value)
