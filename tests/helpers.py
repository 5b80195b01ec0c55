"""Shared helpers for the tests: fixtures, seeded states, case scripts."""
import os

import numpy as np

import shhd_oracle as so

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_cases.npz")


def load_golden():
    from golden.cases import CASES
    data = np.load(GOLDEN)
    out = {}
    for name, script in CASES.items():
        out[name] = dict(script=script, u0=data[f"{name}/u0"], det=data[f"{name}/det"], noise=data[f"{name}/noise"],
                         states=data[f"{name}/states"])
    return out


GOLDEN_INITIAL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_initial.npz")


def load_initial_golden():
    """Initial-condition cases: script, and the reference's initial state or its error message."""
    from golden.cases import IC_CASES
    data = np.load(GOLDEN_INITIAL)
    out = {}
    for name, script in IC_CASES.items():
        err = f"{name}/error"
        out[name] = dict(script=script, u0=None if err in data else data[f"{name}/u0"],
                         error=str(data[err]) if err in data else None)
    return out


def random_state(cfg: so.Config, seed: int, amp: float = 0.05, rho0: float = 1.0, transverse: bool = False) -> np.ndarray:
    """A valid spectral state: active modes only, Hermitian kx = 0 line, smooth spectrum.

    Real-space fluctuations of each field have rms ~ amp; rho has mean rho0.
    """
    g = so.Geometry(cfg)
    rng = np.random.default_rng(seed)
    shape = (cfg.nfields, g.ny, g.hx)
    u = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    decay = 1.0 / (1.0 + g.k2 * (cfg.length[0] / (2 * np.pi)) ** 2 / 16.0)
    u *= np.where(g.active, decay, 0.0)[None]
    u[:, 0, 0] = 0.0
    # real-space rms = sqrt(sum |u|^2 * weight) / N^2; scale each field to amp
    w = np.where(g.gx == 0, 1.0, 2.0)
    for f in range(cfg.nfields):
        rms = np.sqrt((np.abs(u[f]) ** 2 * w).sum()) / g.grid_size
        if rms > 0:
            u[f] *= amp / rms
    if transverse:
        n = cfg.num_order_parameters
        with np.errstate(invalid="ignore", divide="ignore"):
            kdotj = (g.kx * u[n + 1] + g.ky * u[n + 2]) / np.where(g.k2 > 0, g.k2, 1.0)
        u[n + 1] -= g.kx * kdotj
        u[n + 2] -= g.ky * kdotj
    u[0, 0, 0] = rho0 * g.grid_size
    o = so.Oracle(cfg)
    return o.enforce_real_symmetry(u)


def script(grid=(32, 32), length=(32.0, 32.0), dealias="3/2", nop=2, dt=0.01, te="srk3/compressible", cT=1.0,
           fe="phi4", a=-1.0, b=1.0, u=1.0, eta=1.0, zeta=1.0, M=1.0, nonlinear="all", noise=None, extra=""):
    lines = ["dimension 2", f"grid {grid[0]} {grid[1]}", f"length {length[0]} {length[1]}", f"dealias {dealias}",
             f"order_parameters {nop}", f"timestep {dt}", f"time_evolution {te}"]
    if cT is not None:
        lines.append(f"model thermo linear_eos cT {cT}")
    if nop > 0 and fe == "phi4":
        lines.append("model free_energy phi4 " + " ".join(f"a[{i}] {a} b[{i}] {b} u[{i}] {u}" for i in range(nop)))
    elif nop > 0 and fe == "quadratic":
        lines.append("model free_energy quadratic " + " ".join(f"a[{i}] {a}" for i in range(nop)))
    lines.append(f"model transport constant eta {eta} zeta {zeta} " + " ".join(f"M[{i},{i}] {M}" for i in range(nop)))
    if nonlinear:
        lines.append(f"fix 1 {nonlinear} nonlinear on")
    if noise:
        lines.append(f"fix 2 all noise on {noise}")
    if extra:
        lines.append(extra)
    lines.append("run 1")
    return "\n".join(lines) + "\n"


def fp32_transform_rhs(cfg: so.Config, state: np.ndarray) -> np.ndarray:
    """The oracle's RHS with both transforms in single precision (scipy's pocketfft in float32,
    correctly rounded twiddles), everything else in FP64: the error an FP32 transform pipeline
    cannot avoid, to which the engine's FP32 error is compared at large sizes."""
    import scipy.fft as sf
    o = so.Oracle(cfg)
    g = o.geo
    g.backward = lambda f: sf.irfft2(np.asarray(f).astype(np.complex64), s=(g.ny, g.nx), axes=(-2, -1), workers=8).astype(np.float64)
    g.forward = lambda p: sf.rfft2(np.asarray(p).astype(np.float32), axes=(-2, -1), workers=8).astype(np.complex128)
    return o.rhs(state)
