"""Initial states from the reference's `set` commands (host side, numpy) and their device specs.

Every built-in style is restated here and returns the state in the
reference's State layout (complex128 [field, gy, gx <= nx/2]):

  set density uniform value v ............ initial_condition_uniform_density.cc:14-30
  set density gaussian .................. initial_condition_gaussian_density.cc:31-68
  set density sine ...................... initial_condition_sine_density.cc:30-59
  set density equilibrium/gaussian ....... initial_condition_equilibrium_gaussian_density.cc:16-93
  set momentum <x|y|all> uniform value v . initial_condition_uniform_momentum.cc
  set momentum <..> sine ................. initial_condition_sine_momentum.cc:33-62
  set momentum <..> random_vorticity ..... initial_condition_random_vorticity_momentum.cc:58-147
  set momentum <..> equilibrium/gaussian/compressible
                                          initial_condition_equilibrium_gaussian_momentum_compressible.cc:48-112
  set momentum <..> equilibrium/gaussian/incompressible
                                          initial_condition_equilibrium_gaussian_momentum_incompressible.cc:89-115
  set order_parameter <i|all> uniform | gaussian | sine | equilibrium/gaussian
                                          initial_condition_*_order_parameter.cc

Equilibrium styles: u1, u2 = splitmix64(key(seed, channel, gx, ky, draw)) >> 11 / 2^53
(u1 floored at 1e-300), value = sqrt(-2 ln u1) * exp(2 pi i u2); on the kx = 0
line |ky| keys the draw and ky < 0 takes the conjugate.  Random vorticity keys
one phase per mode by (seed, gx, ky) alone.  Every command clears its field
first, and commands apply in the reference's order: density, then momentum,
then order parameter (src/project.h:92-116); an incompressible run then
requires transverse momentum (initial_condition.cc:7-40).

`field_specs` turns the same commands into one spec per field for
`shhd_engine_set_initial_field`, which generates the field on the device;
`initial_state_device` applies them to an engine member.
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

_M64 = (1 << 64) - 1
_PI = 3.14159265358979323846

# device styles (shhd_initial_field.style)
IC_GAUSSIAN_MODES = 0
IC_TRANSVERSE_GAUSSIAN = 1
IC_RANDOM_VORTICITY = 2
IC_BUMP = 3
IC_SINE = 4

_INCOMPRESSIBLE = 1


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return x ^ (x >> np.uint64(31))


def _u32(a: np.ndarray) -> np.ndarray:
    return a.astype(np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)


def _uniform(seed: int, channel: int, gx: np.ndarray, ky: np.ndarray, draw: int) -> np.ndarray:
    key = np.uint64(seed & 0xFFFFFFFF)
    key = key ^ (np.uint64(channel & 0xFFFFFFFF) << np.uint64(48))
    k = np.full(gx.shape, key, dtype=np.uint64)
    k ^= _u32(gx) << np.uint64(32)
    k ^= _u32(ky) << np.uint64(8)
    k ^= np.uint64(draw & 0xFFFFFFFF)
    r = _splitmix64(k)
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _uniform_phase_key(seed: int, gx: np.ndarray, ky: np.ndarray) -> np.ndarray:
    """random_vorticity's key: seed ^ gx << 32 ^ ky (no channel, no draw)."""
    k = np.full(gx.shape, np.uint64(seed & 0xFFFFFFFF), dtype=np.uint64)
    k ^= _u32(gx) << np.uint64(32)
    k ^= _u32(ky)
    r = _splitmix64(k)
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class _Grid:
    def __init__(self, active: Tuple[int, int], grid: Tuple[int, int], length: Tuple[float, float]):
        self.nax, self.nay = active
        self.nx, self.ny = grid
        self.lx, self.ly = length
        self.hx = self.nx // 2 + 1
        gx = np.arange(self.hx)
        gy = np.arange(self.ny)
        sgy = np.where(gy <= self.ny // 2, gy, gy - self.ny)
        self.gx = np.broadcast_to(gx[None, :], (self.ny, self.hx))
        self.sgy = np.broadcast_to(sgy[:, None], (self.ny, self.hx))
        self.kx = 2.0 * _PI * self.gx / length[0]
        self.ky = 2.0 * _PI * self.sgy / length[1]
        self.k2 = self.kx * self.kx + self.ky * self.ky
        self.active = (self.gx < self.nax // 2) & (np.abs(self.sgy) < self.nay // 2)
        self.grid_size = float(self.nx) * float(self.ny)
        self.volume = length[0] * length[1]

    def gaussian_modes(self, seed: int, channel: int) -> np.ndarray:
        phase_ky = np.where(self.gx == 0, np.abs(self.sgy), self.sgy)
        u1 = np.maximum(_uniform(seed, channel, self.gx, phase_ky, 0), 1.0e-300)
        u2 = _uniform(seed, channel, self.gx, phase_ky, 1)
        r = np.sqrt(-2.0 * np.log(u1))
        th = 2.0 * _PI * u2
        v = r * np.cos(th) + 1j * (r * np.sin(th))
        return np.where((self.gx == 0) & (self.sgy < 0), np.conj(v), v)

    def vorticity_velocity(self, n0: float, sigma: float, seed: int) -> Tuple[np.ndarray, np.ndarray]:
        """(u_x, u_y) of the unnormalised random-vorticity shell, zero at k = 0."""
        phase_ky = np.where(self.gx == 0, np.abs(self.sgy), self.sgy)
        n = np.sqrt(self.gx.astype(np.float64) ** 2 + self.sgy.astype(np.float64) ** 2)
        d = (n - n0) / sigma
        env = np.exp(-0.5 * d * d)
        th = 2.0 * _PI * _uniform_phase_key(seed, self.gx, phase_ky)
        om = env * (np.cos(th) + 1j * np.sin(th))
        om = np.where((self.gx == 0) & (self.sgy < 0), np.conj(om), om)
        nz = self.k2 != 0.0
        k2 = np.where(nz, self.k2, 1.0)
        ux = np.where(nz, (1j * (self.ky / k2)) * om, 0.0)
        uy = np.where(nz, -(1j * (self.kx / k2)) * om, 0.0)
        return ux, uy


def _kv(tokens: List[str]) -> Dict[str, str]:
    if len(tokens) % 2:
        raise ValueError("initial-condition arguments must be key-value pairs")
    return dict(zip(tokens[0::2], tokens[1::2]))


def _set_commands(cfg, script_text: str):
    """The `set` lines of a script grouped as (density, momentum, order parameter) commands."""
    n = cfg.num_order_parameters
    dens, mom, psi = [], [], []
    for raw in script_text.splitlines():
        t = raw.split("#", 1)[0].split()
        if len(t) < 3 or t[0] != "set":
            continue
        if t[1] in ("density", "rho"):
            dens.append((t[2], _kv(t[3:])))
        elif t[1] in ("momentum", "j"):
            targets = [0, 1] if t[2] == "all" else [{"x": 0, "0": 0, "y": 1, "1": 1}[t[2]]]
            for d in targets:
                mom.append((d, t[3], _kv(t[4:])))
        elif t[1] in ("order_parameter", "psi"):
            if t[2] == "all" and n <= 0:
                raise ValueError("set order_parameter all requires at least one order parameter.")
            targets = list(range(n)) if t[2] == "all" else [int(t[2])]
            for a in targets:
                psi.append((a, t[3], _kv(t[4:])))
    return dens, mom, psi


def _seed(kv: Dict[str, str]) -> int:
    return int(kv.get("seed", "12345"))


def _sine_args(cfg, what: str, kv: Dict[str, str], base_required: bool) -> Tuple[float, float, int, int]:
    """(base, amplitude, nkx, nky) with the reference's parse checks (initial_condition_sine_*_style.h)."""
    base = float(kv["base"]) if base_required else float(kv.get("base", "0.0"))
    amp = float(kv["amplitude"])
    nkx, nky = int(kv["nkx"]), int(kv.get("nky", "0"))
    if what == "density" and base - abs(amp) < 0.0:
        raise ValueError("set density sine requires base >= abs(amplitude)")
    if nkx < 0 or nkx >= cfg.active_nx // 2:
        raise ValueError(f"set {what} sine requires 0 <= nkx < Nx/2; Nyquist line is fixed to zero")
    if nky <= -(cfg.active_ny // 2) or nky >= cfg.active_ny // 2:
        raise ValueError(f"set {what} sine requires -Ny/2 < nky < Ny/2; Nyquist line is fixed to zero")
    if nkx == 0 and nky == 0:
        raise ValueError(f"set {what} sine requires a nonzero wave number")
    return base, amp, nkx, nky


def _bump_args(cfg, what: str, kv: Dict[str, str]) -> Tuple[float, float, float, float, float, float]:
    """(base, amplitude, x0, y0, sigma_x, sigma_y) with the reference's parse checks."""
    base, amp = float(kv["base"]), float(kv["amplitude"])
    x0, y0 = float(kv["x0"]), float(kv["y0"])
    if "sigma" in kv:
        sx = sy = float(kv["sigma"])
    else:
        sx, sy = float(kv["sigma_x"]), float(kv["sigma_y"])
    if sx <= 0.0 or sy <= 0.0:
        raise ValueError(f"set {what} gaussian requires positive sigma values")
    if what == "density" and base + min(0.0, amp) < 0.0:
        raise ValueError("set density gaussian requires nonnegative density everywhere")
    if cfg.lx <= 0.0 or cfg.ly <= 0.0:
        raise ValueError(f"set {what} gaussian requires positive domain lengths")
    return base, amp, x0, y0, sx, sy


def _vorticity_args(kv: Dict[str, str]) -> Tuple[float, float, float, int]:
    n0, sigma, urms = float(kv["n0"]), float(kv["sigma"]), float(kv["urms"])
    if n0 <= 0.0:
        raise ValueError("set momentum random_vorticity requires positive n0.")
    if sigma <= 0.0:
        raise ValueError("set momentum random_vorticity requires positive sigma.")
    if urms <= 0.0:
        raise ValueError("set momentum random_vorticity requires positive urms.")
    return n0, sigma, urms, _seed(kv)


def _nonnegative_kbt(what: str, style: str, kbt: float) -> float:
    if kbt < 0.0:
        raise ValueError(f"set {what} {style} requires kBT >= 0.")
    return kbt


def _bump(g: _Grid, base: float, amp: float, x0: float, y0: float, sx: float, sy: float) -> np.ndarray:
    pref = amp * g.grid_size * 2.0 * _PI * sx * sy / (g.lx * g.ly)
    env = np.exp(-0.5 * (sx * sx * g.kx * g.kx + sy * sy * g.ky * g.ky))
    ph = -(g.kx * x0 + g.ky * y0)
    v = np.where(g.active, (pref * env) * (np.cos(ph) + 1j * np.sin(ph)), 0.0)
    v[0, 0] += base * g.grid_size
    return v


def _sine(g: _Grid, base: float, amp: float, nkx: int, nky: int) -> np.ndarray:
    v = np.zeros((g.ny, g.hx), dtype=np.complex128)
    v[0, 0] = base * g.grid_size
    pos = complex(0.0, -0.5 * amp * g.grid_size)
    v[nky % g.ny, nkx] = pos
    if nkx == 0 and nky != 0:
        v[(-nky) % g.ny, 0] = pos.conjugate()
    return v


def _reference_density(u: np.ndarray, g: _Grid) -> float:
    return u[0, 0, 0].real / g.grid_size


def check_transverse(cfg, u: np.ndarray) -> None:
    """The incompressible check on the initial momentum (initial_condition.cc:7-40)."""
    g = _Grid((cfg.active_nx, cfg.active_ny), (cfg.nx, cfg.ny), (cfg.lx, cfg.ly))
    n = cfg.num_order_parameters
    jx, jy = u[n + 1], u[n + 2]
    use = g.active & (g.k2 != 0.0)
    viol = np.abs(g.kx * jx + g.ky * jy)
    scale = np.sqrt(g.k2) * np.sqrt(np.abs(jx) ** 2 + np.abs(jy) ** 2)
    if np.any(use & (viol > 1.0e-10 + 1.0e-10 * scale)):
        raise ValueError("incompressible initial momentum must be transverse: k dot j must be zero for every nonzero "
                         "active spectral mode.")


def initial_state(cfg, script_text: str) -> np.ndarray:
    """State from the `set` lines of a script; cfg is a shhd_b200.Config (grid, length, N, mode)."""
    g = _Grid((cfg.active_nx, cfg.active_ny), (cfg.nx, cfg.ny), (cfg.lx, cfg.ly))
    n = cfg.num_order_parameters
    u = np.zeros((n + 3, g.ny, g.hx), dtype=np.complex128)
    dens, mom, psi = _set_commands(cfg, script_text)
    act = g.active
    use = act & (g.k2 != 0.0)
    cell = g.volume / g.grid_size
    for style, kv in dens:
        rho = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            rho[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "gaussian":
            rho = _bump(g, *_bump_args(cfg, "density", kv))
        elif style == "sine":
            rho = _sine(g, *_sine_args(cfg, "density", kv, True))
        elif style == "equilibrium/gaussian":
            kbt = _nonnegative_kbt("density", style, float(kv["kBT"]))
            rho0, cT, seed = float(kv["rho0"]), float(kv["cT"]), _seed(kv)
            if rho0 <= 0.0:
                raise ValueError(f"set density {style} requires rho0 > 0.")
            if cT <= 0.0:
                raise ValueError(f"set density {style} requires cT > 0.")
            rho[0, 0] = rho0 * g.grid_size
            if kbt != 0.0:
                sigma = math.sqrt(kbt * g.grid_size * rho0 / (2.0 * (cT * cT) * cell))
                rho = np.where(use, sigma * g.gaussian_modes(seed, 0), rho)
        else:
            raise NotImplementedError(f"set density {style}")
        u[0] = rho
    for d, style, kv in mom:
        f = n + 1 + d
        m = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            m[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "sine":
            m = _sine(g, *_sine_args(cfg, "momentum", kv, True))
        elif style == "random_vorticity":
            n0, sigma, urms, seed = _vorticity_args(kv)
            ux, uy = g.vorticity_velocity(n0, sigma, seed)
            w = np.where(g.gx == 0, 1.0, 2.0)
            norm = float(np.sum(np.where(act, w * (np.abs(ux) ** 2 + np.abs(uy) ** 2), 0.0)))
            if norm == 0.0:
                raise ValueError("set momentum random_vorticity generated zero velocity field.")
            rho0 = _reference_density(u, g)
            if rho0 == 0.0:
                raise ValueError("set momentum random_vorticity requires nonzero reference density.")
            scale = urms * g.grid_size / math.sqrt(norm)
            m = np.where(act, (rho0 * scale) * (ux if d == 0 else uy), 0.0)
        elif style in ("equilibrium/gaussian/compressible", "equilibrium/gaussian/incompressible"):
            kbt, seed = _nonnegative_kbt("momentum", style, float(kv["kBT"])), _seed(kv)
            if kbt != 0.0:
                rho0 = _reference_density(u, g)
                if rho0 <= 0.0:
                    raise ValueError(f"set momentum {style} requires positive reference density.")
                sigma = math.sqrt(kbt * g.grid_size * rho0 / (2.0 * cell))
                if style.endswith("/compressible"):
                    m = np.where(use, sigma * g.gaussian_modes(seed, d), 0.0)
                else:
                    k = np.sqrt(np.where(use, g.k2, 1.0))
                    comp = -g.ky / k if d == 0 else g.kx / k
                    m = np.where(use, comp * (sigma * g.gaussian_modes(seed, 0)), 0.0)
        else:
            raise NotImplementedError(f"set momentum {style}")
        u[f] = m
    for a, style, kv in psi:
        f = 1 + a
        p = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            p[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "gaussian":
            p = _bump(g, *_bump_args(cfg, "order_parameter", kv))
        elif style == "sine":
            p = _sine(g, *_sine_args(cfg, "order_parameter", kv, False))
        elif style == "equilibrium/gaussian":
            kbt, seed = _nonnegative_kbt("order_parameter", style, float(kv["kBT"])), _seed(kv)
            psi0 = float(kv.get("psi0", "0.0"))
            k0, k2c, k4 = float(kv["k0"]), float(kv.get("k2", "0.0")), float(kv.get("k4", "0.0"))
            p[0, 0] = psi0 * g.grid_size
            if kbt != 0.0:
                coef = k0 + k2c * g.k2 + k4 * g.k2 * g.k2
                if np.any(coef[use] <= 0.0):
                    raise ValueError("set order_parameter equilibrium/gaussian requires positive linear chemical-potential "
                                     "coefficient for every active nonzero mode.")
                with np.errstate(divide="ignore", invalid="ignore"):
                    sigma = np.sqrt(kbt * g.grid_size / (2.0 * coef * cell))
                p = np.where(use, sigma * g.gaussian_modes(seed, a), p)
        else:
            raise NotImplementedError(f"set order_parameter {style}")
        u[f] = p
    if cfg.mode == _INCOMPRESSIBLE:
        check_transverse(cfg, u)
    return u


def _spec(style: int, **kw) -> Dict[str, float]:
    s = dict(style=style, channel=0, seed=0, mean=0.0, s0=0.0, c0=1.0, c2=0.0, c4=0.0, amplitude=0.0, rho0=0.0,
             n0=0.0, sigma=0.0, x0=0.0, y0=0.0, sigma_x=1.0, sigma_y=1.0, nkx=0, nky=0)
    s.update(kw)
    return s


def field_specs(cfg, script_text: str) -> List[Dict[str, float]]:
    """One device spec (the fields of shhd_initial_field) per field: the state `initial_state` builds.

    Every `set` command rewrites its whole field, so the last command on a field decides it; the
    momentum styles read the reference density the density commands left (src/project.h:92-116).
    """
    n = cfg.num_order_parameters
    ng = float(cfg.nx) * float(cfg.ny)
    cell = cfg.lx * cfg.ly / ng
    specs = {f: _spec(IC_GAUSSIAN_MODES) for f in range(n + 3)}
    dens, mom, psi = _set_commands(cfg, script_text)

    def bump(what, kv):
        base, amp, x0, y0, sx, sy = _bump_args(cfg, what, kv)
        return _spec(IC_BUMP, mean=base * ng, amplitude=amp, x0=x0, y0=y0, sigma_x=sx, sigma_y=sy)

    def sine(what, kv, base_required):
        base, amp, nkx, nky = _sine_args(cfg, what, kv, base_required)
        return _spec(IC_SINE, mean=base * ng, amplitude=amp, nkx=nkx, nky=nky)

    for style, kv in dens:
        if style == "uniform":
            specs[0] = _spec(IC_GAUSSIAN_MODES, mean=float(kv["value"]) * ng)
        elif style == "gaussian":
            specs[0] = bump("density", kv)
        elif style == "sine":
            specs[0] = sine("density", kv, True)
        elif style == "equilibrium/gaussian":
            kbt = _nonnegative_kbt("density", style, float(kv["kBT"]))
            rho0, cT = float(kv["rho0"]), float(kv["cT"])
            if rho0 <= 0.0:
                raise ValueError(f"set density {style} requires rho0 > 0.")
            if cT <= 0.0:
                raise ValueError(f"set density {style} requires cT > 0.")
            s0 = kbt * ng * rho0 / (2.0 * (cT * cT) * cell) if kbt != 0.0 else 0.0
            specs[0] = _spec(IC_GAUSSIAN_MODES, seed=_seed(kv), mean=rho0 * ng, s0=s0)
        else:
            raise NotImplementedError(f"set density {style}")
    # the (0, 0) density coefficient each style leaves (the bump adds its own k = 0 value)
    d0 = specs[0]
    if d0["style"] == IC_BUMP:
        rho_00 = d0["amplitude"] * ng * 2.0 * _PI * d0["sigma_x"] * d0["sigma_y"] / (cfg.lx * cfg.ly) + d0["mean"]
    else:
        rho_00 = d0["mean"]
    rho0 = rho_00 / ng
    for d, style, kv in mom:
        f = n + 1 + d
        if style == "uniform":
            specs[f] = _spec(IC_GAUSSIAN_MODES, mean=float(kv["value"]) * ng)
        elif style == "sine":
            specs[f] = sine("momentum", kv, True)
        elif style == "random_vorticity":
            n0, sigma, urms, seed = _vorticity_args(kv)
            specs[f] = _spec(IC_RANDOM_VORTICITY, channel=d, seed=seed, amplitude=urms, rho0=rho0, n0=n0, sigma=sigma)
        elif style in ("equilibrium/gaussian/compressible", "equilibrium/gaussian/incompressible"):
            kbt = _nonnegative_kbt("momentum", style, float(kv["kBT"]))
            s0 = 0.0
            if kbt != 0.0:
                if rho0 <= 0.0:
                    raise ValueError(f"set momentum {style} requires positive reference density.")
                s0 = kbt * ng * rho0 / (2.0 * cell)
            if style.endswith("/compressible"):
                specs[f] = _spec(IC_GAUSSIAN_MODES, seed=_seed(kv), channel=d, s0=s0)
            else:
                specs[f] = _spec(IC_TRANSVERSE_GAUSSIAN, seed=_seed(kv), channel=d, s0=s0)
        else:
            raise NotImplementedError(f"set momentum {style}")
    for a, style, kv in psi:
        f = 1 + a
        if style == "uniform":
            specs[f] = _spec(IC_GAUSSIAN_MODES, mean=float(kv["value"]) * ng)
        elif style == "gaussian":
            specs[f] = bump("order_parameter", kv)
        elif style == "sine":
            specs[f] = sine("order_parameter", kv, False)
        elif style == "equilibrium/gaussian":
            kbt = _nonnegative_kbt("order_parameter", style, float(kv["kBT"]))
            psi0 = float(kv.get("psi0", "0.0"))
            k0, k2c, k4 = float(kv["k0"]), float(kv.get("k2", "0.0")), float(kv.get("k4", "0.0"))
            s0 = kbt * ng / (2.0 * cell) if kbt != 0.0 else 0.0
            specs[f] = _spec(IC_GAUSSIAN_MODES, seed=_seed(kv), channel=a, mean=psi0 * ng, s0=s0, c0=k0, c2=k2c, c4=k4)
        else:
            raise NotImplementedError(f"set order_parameter {style}")
    return [specs[f] for f in range(n + 3)]


def initial_state_device(engine, script_text: str, member: int = 0) -> None:
    """Write the state of a script's `set` lines into one member of `engine`, generated on the device.

    The fields are those of `initial_state` (one kernel per field; no state crosses PCIe); an
    incompressible configuration then has its momentum checked for transversality in FP64.
    """
    cfg = engine.cfg
    specs = field_specs(cfg, script_text)
    for f, s in enumerate(specs):
        engine.set_initial_field(member, f, s)
    if cfg.mode == _INCOMPRESSIBLE:
        n = cfg.num_order_parameters
        engine.check_transverse(specs[n + 1], specs[n + 2])
