"""Yokota-Green-Kubo stress measure on the device (GPU) against the FP64 restatement.

The oracle restates the reference's momentum flux pi_xy (fcalculator.cc,
buffer_flux.cc, stage weights of time_integrator_srk3_*.h) and the measure's
block accounting (measure_yokota_green_kubo.cc:128-190) on the same Philox
noise, and both run the same trajectory.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import random_state, script

pytestmark = pytest.mark.gpu

COMP = script(grid=(24, 24), length=(48.0, 48.0), nop=1, dt=0.01, eta=0.5, zeta=0.3, noise="kBT 0.002 seed 6")
INCOMP = script(grid=(24, 32), length=(48.0, 64.0), nop=0, dt=0.01, te="srk3/incompressible", cT=None, eta=0.3, zeta=0.0,
                nonlinear="momentum", noise="kBT 0.001 seed 8")
EULER = script(grid=(24, 24), length=(48.0, 48.0), nop=0, dt=0.004, te="euler/compressible", eta=0.5, zeta=0.5,
               noise="kBT 0.002 seed 9")


def _oracle_gk(text, u0, nsteps, nevery, nblock, selection):
    cfg = so.parse_script(text)
    o = so.Oracle(cfg)
    gk = so.GreenKubo(cfg, nevery, nblock, selection)
    u = u0
    for _ in range(nsteps):
        u, flux = o.step_with_flux(u, "philox")
        gk.observe(flux)
    return gk, u


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name,text,selection", [("comp", COMP, "diagonal"), ("incomp", INCOMP, "all"), ("euler", EULER, "all")])
def test_green_kubo_matches_restatement(precision, name, text, selection):
    import shhd_b200 as sb
    cfg = so.parse_script(text)
    u0 = random_state(cfg, seed=4, transverse=(cfg.mode == "incompressible"))
    nevery, nblock, nsteps = 2, 6, 14
    gk, uref = _oracle_gk(text, u0, nsteps, nevery, nblock, selection)
    c = sb.config_from_script(text)
    c.precision = precision
    with sb.Engine(c) as eng:
        eng.set_state(u0)
        eng.gk_enable(nevery, nblock, selection)
        assert eng.gk_modes == gk.modes
        eng.step(5)
        eng.step(nsteps - 5)
        sums, blocks = eng.gk_read()
        u = eng.get_state()
    assert blocks == gk.nsample == nsteps // nblock
    tol = 1e-10 if precision == 0 else 2e-4
    assert so.rel_l2(u, uref) < (1e-12 if precision == 0 else 1e-5)
    scale = np.abs(gk.sums).max()
    assert scale > 0
    assert np.abs(sums - gk.sums).max() <= tol * scale, (name, precision, np.abs(sums - gk.sums).max() / scale)


@pytest.mark.parametrize("precision", [0, 1])
def test_autotune_mid_run_leaves_the_measure_intact(precision):
    """The autotuner's trial steps run the measure's taps; it restores their accumulators with the
    state, so that an autotune in the middle of a block changes no sum."""
    import shhd_b200 as sb
    cfg = so.parse_script(COMP)
    u0 = random_state(cfg, seed=14)
    nevery, nblock, nsteps = 2, 6, 14
    gk, uref = _oracle_gk(COMP, u0, nsteps, nevery, nblock, "diagonal")
    c = sb.config_from_script(COMP)
    c.precision = precision
    with sb.Engine(c) as eng:
        eng.set_state(u0)
        eng.gk_enable(nevery, nblock, "diagonal")
        eng.step(5)                    # inside the first block of 6
        eng.autotune(2)
        eng.step(nsteps - 5)
        sums, blocks = eng.gk_read()
        u = eng.get_state()
    assert blocks == gk.nsample
    assert so.rel_l2(u, uref) < (1e-12 if precision == 0 else 1e-5)
    tol = 1e-10 if precision == 0 else 2e-4
    assert np.abs(sums - gk.sums).max() <= tol * np.abs(gk.sums).max()


def test_green_kubo_rejects_what_the_reference_rejects():
    import shhd_b200 as sb
    quiet = script(grid=(24, 24), length=(48.0, 48.0), nop=1, dt=0.01, te="srk3/quiescent", cT=None, eta=0.0, zeta=0.0,
                   nonlinear=None, noise="kBT 0.01 seed 1")
    with sb.Engine(sb.config_from_script(quiet)) as eng:
        with pytest.raises(sb.ShhdError):
            eng.gk_enable(2, 6)
    with sb.Engine(sb.config_from_script(COMP)) as eng:
        with pytest.raises(sb.ShhdError):
            eng.gk_enable(4, 6)      # nblock not a multiple of nevery
