"""C ABI library: loads, exports what include/shhd_b200.h declares, and its
host-only input-script front end agrees with the reference grammar (CPU)."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "spectral-hohenberg-halperin-dynamics-2d_b200")
HEADER = os.path.join(ROOT, "include", "shhd_b200.h")
LIB = os.path.join(PKG, "lib", "libshhd_b200.so")


def _ensure_built():
    if not os.path.exists(LIB):
        subprocess.run(["make", "-C", PKG], check=True, capture_output=True)


_ensure_built()
import shhd_b200 as sb  # noqa: E402
import shhd_oracle as so  # noqa: E402
from helpers import load_golden, script  # noqa: E402


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(shhd_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(LIB)
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(sb.EXPORTED)


def test_library_is_sm100a_native():
    out = subprocess.run(["/usr/local/cuda/bin/cuobjdump", "--list-elf", LIB], capture_output=True, text=True).stdout
    assert "sm_100a" in out


def test_defaults_follow_reference():
    c = sb.default_config()
    assert (c.active_nx, c.active_ny, c.nx, c.ny) == (128, 128, 128, 128)
    assert c.dt == 0.005 and c.mode == sb.COMPRESSIBLE and c.integrator == sb.SRK3
    assert c.noise_seed == 12345 and c.kBT == 1.0 and c.chi == 1.0
    assert abs(c.lx - 2 * np.pi) < 1e-15


@pytest.mark.parametrize("name", sorted(load_golden()))
def test_script_parser_matches_oracle(name):
    text = load_golden()[name]["script"]
    c = sb.config_from_script(text)
    o = so.parse_script(text)
    assert (c.active_nx, c.active_ny) == o.active
    assert (c.nx, c.ny) == o.grid
    assert (c.lx, c.ly) == o.length
    assert c.dt == o.dt
    assert c.num_order_parameters == o.num_order_parameters
    assert ["compressible", "incompressible", "quiescent"][c.mode] == o.mode
    assert ["euler", "srk3"][c.integrator] == o.integrator
    for a in range(o.num_order_parameters):
        assert c.mobility[a] == o.mobility[a]
        assert c.mu_k0[a] == o.mu_k0(a) and c.mu_k2[a] == o.mu_k2(a)
        assert c.mu_u3[a] == (o.phi4_u[a] if o.free_energy == "phi4" else 0.0)
    assert (c.eta, c.zeta, c.cT) == (o.eta, o.zeta, o.cT)
    assert bool(c.momentum_advection) == o.momentum_advection
    assert bool(c.order_parameter_advection) == o.order_parameter_advection
    assert bool(c.noise_momentum) == o.noise_momentum
    assert bool(c.noise_order_parameter) == o.noise_order_parameter
    assert c.noise_seed == o.noise_seed and c.kBT == o.kBT and c.chi == o.chi
    assert c.n_sine_forces == len(o.sine_forces) and c.n_gradient_forces == len(o.gradient_forces)


@pytest.mark.parametrize("text, message", [
    ("grid 15 16\n", "grid must be even."),
    ("foo 1\n", "Unknown command: foo"),
    ("dimension 3\n", "This solver only supports dimension 2."),
    ("dealias three\n", "unknown dealias rule: three"),
    ("grid 16 16\nmodel transport constant eta -1\n", "model transport constant requires nonnegative eta."),
    ("order_parameters 1\nmodel transport constant M[0,0] 1\nmodel free_energy phi4 u[0] -1\n",
     "model free_energy phi4 requires nonnegative u[0]."),
    ("order_parameters 1\nmodel transport constant M[0,1] 1\n", "model transport constant mobility index out of range: M[0,1]"),
    ("time_evolution srk3/quiescent\nmodel transport constant eta 0\nfix 1 momentum nonlinear on\n",
     "quiescent time evolution cannot use momentum nonlinear advection."),
    ("grid 16 16\nmodel transport constant eta 1\nfix 1 momentum force/sine on component x axis y nk 8 amplitude 1\n",
     "fix force/sine requires nk < active_N_axis/2."),
    ("model transport constant eta 1\nfix 1 all noise on kBT -1\n", "fix noise requires nonnegative kBT."),
    ("grid 16 16\n", "model transport must be specified"),
    ("time_evolution rk4/compressible\nmodel transport constant eta 1\n", "unknown time_evolution type: rk4/compressible"),
    ("model transport constant eta 1\nrun 10\nfix 1 all nonlinear on\n", "fix must be specified before run or measure commands"),
])
def test_script_errors_follow_reference(text, message):
    with pytest.raises(sb.ShhdError) as ei:
        sb.config_from_script(text)
    assert ei.value.code == sb.SHHD_EINVAL
    assert str(ei.value) == message


def test_dealias_rules_and_quiescent_noise():
    c = sb.config_from_script(script(grid=(64, 32), dealias="3/2"))
    assert (c.nx, c.ny) == (96, 48)
    c = sb.config_from_script(script(grid=(64, 32), dealias="two"))
    assert (c.nx, c.ny) == (128, 64)
    c = sb.config_from_script(script(grid=(64, 32), dealias="none"))
    assert (c.nx, c.ny) == (64, 32)
    c = sb.config_from_script(script(te="srk3/quiescent", nonlinear=None, cT=None, noise="kBT 0.1"))
    assert c.noise_momentum == 0 and c.noise_order_parameter == 1


def test_reference_checker_parses_the_same_scripts():
    """When the reference checker is built, its parse of each golden script
    gives the same compute grid and field count as the C ABI front end."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so")
    if not os.path.exists(ref):
        pytest.skip("oracle/_ref not built (needs the reference sources)")
    lib = ctypes.CDLL(ref)
    lib.shref_create.restype = ctypes.c_void_p
    for name, c in load_golden().items():
        h = ctypes.c_void_p(lib.shref_create(c["script"].encode()))
        info = (ctypes.c_long * 10)()
        dinfo = (ctypes.c_double * 4)()
        lib.shref_info(h, info, dinfo)
        cfg = sb.config_from_script(c["script"])
        assert (info[0], info[1], info[2], info[3]) == (cfg.nx, cfg.ny, cfg.active_nx, cfg.active_ny)
        assert info[4] == cfg.num_order_parameters + 3
        assert info[9] == cfg.mode
        lib.shref_destroy(h)
