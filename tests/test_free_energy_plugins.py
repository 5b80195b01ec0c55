"""Free-energy plugin styles: the compile-time registry (include/shhd_b200_free_energy.cuh,
csrc/free_energy_plugins.h) that stands in for the reference's FreeEnergyRegistry
(src/model_free_energy_registry.h:65-85) on the hot path.

CPU: the library lists its styles and their keys, and the script front end parses a style's
keys with the reference's error behaviour.  GPU: the engine's RHS, trajectories and energy
measure with a plugin style against the FP64 oracle's restatement of the same style, in every
kernel family and both precisions; coupled_phi4 with g = 0 is phi4 exactly.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script


def _with_style(text: str, nop: int, style: str, extra: str) -> str:
    old = "model free_energy phi4 " + " ".join(f"a[{i}] -1.0 b[{i}] 1.0 u[{i}] 1.0" for i in range(nop))
    assert old in text
    lin = " ".join(f"a[{i}] -1.0 b[{i}] 1.0" for i in range(nop))
    return text.replace(old, f"model free_energy {style} {lin} {extra}")


BASE = script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01)
COUPLED = _with_style(BASE, 2, "coupled_phi4", "u[0] 1.0 u[1] 0.5 g 0.7")
PHI6 = _with_style(BASE, 2, "phi6", "u[0] 1.0 u[1] 0.5 w[0] 0.3 w[1] 0.2")


def test_library_lists_its_plugin_styles():
    import shhd_b200 as sb
    styles = sb.free_energy_plugins()
    assert styles["coupled_phi4"] == (1, ["u[]", "g"])
    assert styles["phi6"] == (2, ["u[]", "w[]"])


def test_script_front_end_parses_plugin_keys():
    import shhd_b200 as sb
    c = sb.config_from_script(COUPLED)
    assert c.free_energy == 3 and c.fe_plugin == 1
    assert list(c.fe_param[0])[:2] == [1.0, 0.5] and c.fe_param[1][0] == 0.7
    assert list(c.mu_k0)[:2] == [-1.0, -1.0] and list(c.mu_k2)[:2] == [1.0, 1.0]
    c6 = sb.config_from_script(PHI6)
    assert c6.fe_plugin == 2 and list(c6.fe_param[1])[:2] == [0.3, 0.2]
    bad = {
        "g 0.7": ("u[2] 1", "model free_energy coupled_phi4 coefficient index out of range: u[2]"),
        "u[1] 0.5 g": ("u[1] 0.5 h", "unknown coupled_phi4 free energy coefficient: h"),
    }
    for old, (new, msg) in bad.items():
        with pytest.raises(sb.ShhdError) as ei:
            sb.config_from_script(COUPLED.replace(old, new))
        assert ei.value.code == sb.SHHD_EINVAL and msg in str(ei.value)
    with pytest.raises(sb.ShhdError) as ei:
        sb.config_from_script(COUPLED.replace("coupled_phi4", "no_such_style"))
    assert "Unknown free energy type: no_such_style" in str(ei.value)


def _engine(sb, text, precision, family=-1, batch=1):
    cfg = sb.config_from_script(text)
    cfg.precision = precision
    cfg.batch = batch
    e = sb.Engine(cfg)
    e.set_family(family)
    return e


CASES = {
    "coupled_n2_96": COUPLED,
    "phi6_n2_96": PHI6,
    "coupled_n3_quiescent": _with_style(script(grid=(64, 32), length=(128.0, 64.0), nop=3, dt=0.02, te="srk3/quiescent", cT=None,
                                               eta=0.0, zeta=0.0, nonlinear=None), 3, "coupled_phi4", "u[0] 1 u[1] 1 u[2] 1 g 1"),
    "coupled_n1_incomp": _with_style(script(grid=(64, 64), length=(128.0, 128.0), nop=1, dt=0.01, te="srk3/incompressible",
                                            cT=None, eta=0.05, zeta=0.0), 1, "coupled_phi4", "u[0] 2 g 5"),
    "phi6_n2_1536": _with_style(script(grid=(1024, 64), length=(2048.0, 128.0), nop=2, dt=0.01), 2, "phi6",
                                "u[0] 1 u[1] 1 w[0] 0.5 w[1] 0.5"),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_plugin_rhs_matches_oracle(name):
    import shhd_b200 as sb
    text = CASES[name]
    cfg = so.parse_script(text)
    u = random_state(cfg, seed=61, amp=0.3, transverse=cfg.mode == "incompressible")
    want = so.Oracle(cfg).rhs(u)
    with _engine(sb, text, sb.FP64) as e:
        e.set_state(u)
        err64 = so.rel_l2(e.rhs(), want)
    errs = {}
    for fam in (0, 1, 3):
        with _engine(sb, text, sb.FP32, fam) as e:
            e.set_state(u)
            errs[fam, e.family] = so.rel_l2(e.rhs(), want)
    print(f"{name}: FP64 {err64:.2e}, FP32 (requested, used family): {errs}")
    assert err64 < 1e-12
    assert all(v < 1e-5 for v in errs.values())


@pytest.mark.gpu
def test_coupled_phi4_without_coupling_is_phi4():
    import shhd_b200 as sb
    text = _with_style(BASE, 2, "coupled_phi4", "u[0] 1.0 u[1] 1.0 g 0")
    cfg = so.parse_script(BASE)
    u = random_state(cfg, seed=62, amp=0.3)
    with _engine(sb, BASE, sb.FP64, 0) as e, _engine(sb, text, sb.FP64, 0) as p:
        e.set_state(u)
        p.set_state(u)
        assert np.array_equal(e.rhs(), p.rhs())


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_plugin_trajectory_and_energies(precision):
    import shhd_b200 as sb
    text = COUPLED.replace("run 1", "fix 9 all noise on seed 4 kBT 0.001\nrun 1")
    cfg = so.parse_script(text)
    u = random_state(cfg, seed=63, amp=0.3)
    o = so.Oracle(cfg)
    ref = u
    for _ in range(5):
        ref = o.step(ref, "philox")
    with _engine(sb, text, precision) as e:
        e.set_state(u)
        e.step(5)
        got = e.get_state()
        assert so.rel_l2(got, ref) < (1e-12 if precision == 0 else 1e-5)
        want = so.time_series_energies(cfg, got)
        have = e.time_series_energies()
    for k in ("E_T", "E_psi"):
        assert abs(have[k] - want[k]) <= (1e-10 if precision == 0 else 1e-5) * abs(want[k]), (k, have[k], want[k])
