"""The reference-side drop-in B200FluidSolver (include/shhd_b200_fluid_solver.hpp): FluidSolver's
constructor arguments (Params, Domain2D and the three model objects the reference built from
the script) and its step(State&, double), compiled against the reference's own headers into
oracle/_ref/libshhd_dropin.so by the build.

CPU: the configuration the drop-in derives from the reference's Params and model objects equals
the one shhd_config_from_script reads from the same script, for every golden case.
GPU: the reference's own initial State advanced through B200FluidSolver::step matches the
reference's solver (the CPU checker) on noise-free runs, in each host-synchronisation mode.
"""
import ctypes
import os

import numpy as np
import pytest

import shhd_oracle as so
from helpers import script

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "libshhd_dropin.so")
REF = os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so")

needs_dropin = pytest.mark.skipif(not os.path.exists(DROPIN), reason="drop-in harness not built (oracle/_ref)")


def _lib():
    lib = ctypes.CDLL(DROPIN)
    lib.dropin_last_error.restype = ctypes.c_char_p
    lib.dropin_run.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t]
    lib.dropin_config_matches.argtypes = [ctypes.c_char_p]
    return lib


DETERMINISTIC = {
    "compressible_phi4_n2": script(grid=(64, 64), length=(128.0, 128.0), nop=2, dt=0.01,
                                   extra="set density equilibrium/gaussian kBT 1e-3 rho0 1 cT 1 seed 1\n"
                                         "set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 2\n"
                                         "set order_parameter all equilibrium/gaussian seed 7 kBT 0.01 k0 1 k2 0"),
    "incompressible_n1": script(grid=(64, 32), length=(64.0, 32.0), nop=1, dt=0.01, te="srk3/incompressible", cT=None, eta=0.2,
                                zeta=0.0, extra="set density uniform value 1.0\n"
                                                "set momentum all equilibrium/gaussian/incompressible kBT 1e-3 seed 3\n"
                                                "set order_parameter all equilibrium/gaussian seed 2 kBT 0.01 k0 1 k2 0"),
    "quiescent_quadratic_n2": script(grid=(48, 48), length=(96.0, 96.0), nop=2, dt=0.02, te="euler/quiescent", cT=None, eta=0.0,
                                     zeta=0.0, nonlinear=None, fe="quadratic", a=0.5,
                                     extra="set density uniform value 1.0\n"
                                           "set order_parameter all equilibrium/gaussian seed 4 kBT 0.1 k0 1 k2 1"),
    "compressible_forced": script(grid=(32, 32), length=(64.0, 64.0), nop=1, dt=0.01,
                                  extra="fix 3 momentum force/sine on component x axis y nk 1 amplitude 0.01\n"
                                        "fix 4 order_parameter force/gradient on component 0 direction x amplitude 0.02\n"
                                        "set density uniform value 1.0\n"
                                        "set momentum all equilibrium/gaussian/compressible kBT 1e-3 seed 5"),
}


@needs_dropin
def test_config_from_params_and_models_matches_the_script():
    from golden.cases import CASES
    lib = _lib()
    texts = dict(DETERMINISTIC)
    texts.update({f"golden_{k}": v for k, v in CASES.items()})
    for name, text in texts.items():
        rc = lib.dropin_config_matches(text.encode())
        assert rc == 1, f"{name}: {lib.dropin_last_error().decode()}"


def _reference_steps(text, nsteps):
    lib = ctypes.CDLL(REF)
    lib.shref_create.restype = ctypes.c_void_p
    lib.shref_last_error.restype = ctypes.c_char_p
    h = ctypes.c_void_p(lib.shref_create(text.encode()))
    assert h.value, lib.shref_last_error().decode()
    info = (ctypes.c_long * 10)()
    dinfo = (ctypes.c_double * 4)()
    lib.shref_info(h, info, dinfo)
    shape = (info[4], info[1], info[0] // 2 + 1)
    noise = np.zeros((2,) + shape, complex)
    for _ in range(nsteps):
        assert lib.shref_step(h, 1, noise.ctypes.data_as(ctypes.c_void_p)) == 0
    u = np.zeros(shape, complex)
    lib.shref_get_state(h, u.ctypes.data_as(ctypes.c_void_p))
    lib.shref_destroy(h)
    return u


@pytest.mark.gpu
@needs_dropin
@pytest.mark.parametrize("name", sorted(DETERMINISTIC))
def test_drop_in_steps_match_the_reference(name):
    text = DETERMINISTIC[name]
    nsteps = 4
    want = _reference_steps(text, nsteps)
    lib = _lib()
    for precision, tol in ((0, 1e-12), (1, 1e-5)):
        for sync in (0, 1, 2):
            got = np.zeros(want.shape, complex)
            rc = lib.dropin_run(text.encode(), precision, sync, nsteps, got.ctypes.data_as(ctypes.c_void_p), got.size * 2)
            assert rc == 0, lib.dropin_last_error().decode()
            err = so.rel_l2(got, want)
            assert err < tol, f"{name} precision {precision} host sync {sync}: rel L2 {err:.3e}"
