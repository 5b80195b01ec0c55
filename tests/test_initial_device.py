"""Initial conditions generated on the device (shhd_engine_set_initial_field).

CPU: `field_specs` maps each field's last `set` line to one device spec; a
numpy evaluation of those specs (the device kernel's arithmetic restated)
reproduces the reference's own initial states for every style, so the mapping
is pinned without a GPU.

GPU: the device states match the reference's initial states to 1e-13 relative
L2 in FP64 engines (the device's exp/log/sin/cos differ from the host's by an
ulp or two) and to 1e-6 in FP32 engines (one rounding per component), with
the (0, 0) coefficients exact; the reference's refusals come back as the same
messages; random-vorticity norms are summed in a fixed order, so repeated
generation is bitwise identical.
"""
import math

import numpy as np
import pytest

import shhd_oracle as so
from helpers import load_golden, load_initial_golden, script

CASES = load_golden()
IC_CASES = load_initial_golden()
STATES = {**{n: c for n, c in CASES.items()}, **{n: c for n, c in IC_CASES.items() if c["error"] is None}}
ERRORS = {n: c for n, c in IC_CASES.items() if c["error"] is not None}
PI = 3.14159265358979323846


def _evaluate(cfg, specs):
    """The state the specs describe, on the host (numpy restatement of ic_value)."""
    from shhd_b200 import initial as ini
    g = ini._Grid((cfg.active_nx, cfg.active_ny), (cfg.nx, cfg.ny), (cfg.lx, cfg.ly))
    u = np.zeros((len(specs), g.ny, g.hx), dtype=np.complex128)
    use = g.active & (g.k2 != 0.0)
    w = np.where(g.gx == 0, 1.0, 2.0)
    for f, s in enumerate(specs):
        st = s["style"]
        if st == ini.IC_GAUSSIAN_MODES:
            if s["s0"] != 0.0:
                with np.errstate(divide="ignore", invalid="ignore"):
                    sigma = np.sqrt(s["s0"] / (s["c0"] + s["c2"] * g.k2 + s["c4"] * g.k2 * g.k2))
                u[f] = np.where(use, sigma * g.gaussian_modes(s["seed"], s["channel"]), 0.0)
            u[f, 0, 0] = s["mean"]
        elif st == ini.IC_TRANSVERSE_GAUSSIAN:
            if s["s0"] != 0.0:
                k = np.sqrt(np.where(use, g.k2, 1.0))
                comp = -g.ky / k if s["channel"] == 0 else g.kx / k
                u[f] = np.where(use, comp * (math.sqrt(s["s0"]) * g.gaussian_modes(s["seed"], 0)), 0.0)
        elif st == ini.IC_RANDOM_VORTICITY:
            ux, uy = g.vorticity_velocity(s["n0"], s["sigma"], s["seed"])
            norm = float(np.sum(np.where(g.active, w * (np.abs(ux) ** 2 + np.abs(uy) ** 2), 0.0)))
            factor = s["rho0"] * (s["amplitude"] * g.grid_size / math.sqrt(norm))
            u[f] = np.where(g.active, factor * (ux if s["channel"] == 0 else uy), 0.0)
        elif st == ini.IC_BUMP:
            pref = s["amplitude"] * g.grid_size * 2.0 * PI * s["sigma_x"] * s["sigma_y"] / (cfg.lx * cfg.ly)
            u[f] = ini._bump(g, 0.0, s["amplitude"], s["x0"], s["y0"], s["sigma_x"], s["sigma_y"])
            u[f, 0, 0] = pref + s["mean"]
        elif st == ini.IC_SINE:
            u[f] = ini._sine(g, 0.0, s["amplitude"], s["nkx"], s["nky"])
            u[f, 0, 0] = s["mean"]
    return u


@pytest.mark.parametrize("name", sorted(STATES))
def test_specs_reproduce_reference_states(name):
    import shhd_b200 as sb
    from shhd_b200.initial import field_specs
    c = STATES[name]
    cfg = sb.config_from_script(c["script"])
    u = _evaluate(cfg, field_specs(cfg, c["script"]))
    assert so.rel_l2(u, c["u0"]) < 1e-14


def test_specs_last_command_wins_and_missing_fields_are_zero():
    import shhd_b200 as sb
    from shhd_b200.initial import IC_GAUSSIAN_MODES, IC_SINE, field_specs, initial_state
    text = script(grid=(32, 32), nop=2) + "\n".join([
        "",
        "set density uniform value 2.0",
        "set density equilibrium/gaussian kBT 1e-3 rho0 1.5 cT 1 seed 3",
        "set order_parameter 1 equilibrium/gaussian seed 2 kBT 1 k0 4 k2 1",
        "set order_parameter 1 uniform value 0.25",
        "set momentum x equilibrium/gaussian/compressible kBT 1e-3 seed 6",
        "set momentum y sine base 0 amplitude 0.1 nkx 1 nky 2",
    ])
    cfg = sb.config_from_script(text)
    specs = field_specs(cfg, text)
    assert so.rel_l2(_evaluate(cfg, specs), initial_state(cfg, text)) < 1e-14
    ng = cfg.nx * cfg.ny                            # the 3/2-padded transform grid, 48 x 48
    cell = cfg.lx * cfg.ly / ng
    assert specs[1]["style"] == IC_GAUSSIAN_MODES and (specs[1]["mean"], specs[1]["s0"]) == (0.0, 0.0)  # never set
    assert (specs[2]["mean"], specs[2]["s0"]) == (0.25 * ng, 0.0)   # the uniform command came last
    assert specs[4]["style"] == IC_SINE
    assert math.isclose(specs[3]["s0"], 1e-3 * ng * 1.5 / (2.0 * cell))  # momentum x reads rho0 = 1.5


def test_default_seed_is_the_reference_default():
    import shhd_b200 as sb
    from shhd_b200.initial import field_specs
    text = script(grid=(16, 16), nop=1) + "\nset order_parameter all equilibrium/gaussian kBT 1 k0 2\n"
    assert field_specs(sb.config_from_script(text), text)[1]["seed"] == 12345


def _device_state(sb, cfg, text, precision, batch=1, member=0):
    from shhd_b200.initial import initial_state_device
    c = cfg.copy()
    c.precision = precision
    c.batch = batch
    eng = sb.Engine(c)
    initial_state_device(eng, text, member=member)
    return eng


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(STATES))
def test_device_initial_state_matches_reference(name, precision):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    c = STATES[name]
    cfg = sb.config_from_script(c["script"])
    cfg.precision = precision
    cfg.batch = 2
    with sb.Engine(cfg) as eng:
        other = np.zeros_like(c["u0"])
        eng.set_state(c["u0"] * 0.5, member=0)   # the generated member is overwritten everywhere
        eng.set_state(other, member=1)
        initial_state_device(eng, c["script"], member=0)
        got = eng.get_state(0)
        tol = 1e-13 if precision == 0 else 1e-6
        assert so.rel_l2(got, c["u0"]) < tol
        if precision == 0:
            assert np.allclose(got[:, 0, 0], c["u0"][:, 0, 0], rtol=1e-14, atol=0.0)
        else:  # FP32 engines keep the evolved fields' k = 0 coefficients in FP64
            assert np.allclose(got[:, 0, 0], c["u0"][:, 0, 0], rtol=1e-7, atol=0.0)
        assert np.array_equal(eng.get_state(1), other)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(ERRORS))
def test_device_initial_state_refuses_like_the_reference(name):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state_device
    c = ERRORS[name]
    cfg = sb.config_from_script(c["script"])
    with sb.Engine(cfg) as eng:
        with pytest.raises((ValueError, sb.ShhdError)) as ei:
            initial_state_device(eng, c["script"])
        assert str(ei.value) == c["error"]


@pytest.mark.gpu
def test_device_initial_state_steps_like_the_uploaded_state():
    import shhd_b200 as sb
    c = CASES["srk3_compressible_n2"]
    cfg = sb.config_from_script(c["script"])
    with _device_state(sb, cfg, c["script"], 0) as a, sb.Engine(cfg) as b:
        b.set_state(c["u0"])
        a.step(3)
        b.step(3)
        assert so.rel_l2(a.get_state(), b.get_state()) < 1e-12


@pytest.mark.gpu
def test_device_initial_state_is_reproducible():
    import shhd_b200 as sb
    c = IC_CASES["vorticity_on_bump_density"]
    cfg = sb.config_from_script(c["script"])
    with _device_state(sb, cfg, c["script"], 0) as a, _device_state(sb, cfg, c["script"], 0) as b:
        assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["compressible", "incompressible"])
def test_device_initial_state_full_size(mode):
    """1024^2 grid (1536^2 transforms): every style family at the benchmark size."""
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state
    if mode == "compressible":
        text = script(grid=(1024, 1024), length=(2048.0, 2048.0), nop=2, dt=0.01) + "\n".join([
            "",
            "set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 11",
            "set momentum x equilibrium/gaussian/compressible kBT 1e-3 seed 12",
            "set momentum y sine base 0.01 amplitude 0.02 nkx 5 nky -7",
            "set order_parameter 0 equilibrium/gaussian seed 13 kBT 0.04 k0 2 k2 1",
            "set order_parameter 1 gaussian base 0 amplitude 0.5 x0 700 y0 1100 sigma_x 40 sigma_y 90",
        ])
    else:
        text = script(grid=(1024, 1024), length=(2048.0, 2048.0), nop=1, dt=0.01, te="srk3/incompressible", cT=None,
                      eta=0.05, zeta=0.0, nonlinear="momentum") + "\n".join([
            "",
            "set density gaussian base 1 amplitude 0.1 x0 1000 y0 500 sigma 300",
            "set momentum all random_vorticity n0 20 sigma 4 urms 0.2 seed 8",
            "set order_parameter all sine amplitude 0.3 nkx 0 nky 9",
        ])
    cfg = sb.config_from_script(text)
    with _device_state(sb, cfg, text, 0) as eng:
        assert so.rel_l2(eng.get_state(), initial_state(cfg, text)) < 1e-13
