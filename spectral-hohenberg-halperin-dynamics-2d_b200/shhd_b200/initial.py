"""Initial states from the reference's `set` commands (host side, numpy).

The reference's equilibrium initial conditions draw every active mode from a
counter-based generator, so a state is reproducible from (seed, channel, mode)
alone; this module restates those styles and returns the state in the
reference's State layout (complex128 [field, gy, gx <= nx/2]):

  set density uniform value v ............ initial_condition_uniform_density.cc:14-30
  set density equilibrium/gaussian ....... initial_condition_equilibrium_gaussian_density.cc:16-93
  set momentum <x|y|all> uniform value v . initial_condition_uniform_momentum.cc
  set momentum <..> equilibrium/gaussian/compressible
                                          initial_condition_equilibrium_gaussian_momentum_compressible.cc:48-112
  set order_parameter <i|all> uniform value v
  set order_parameter <i|all> equilibrium/gaussian
                                          initial_condition_equilibrium_gaussian_order_parameter.cc:16-108

Per mode: u1, u2 = splitmix64(key(seed, channel, gx, ky, draw)) >> 11 / 2^53
(u1 floored at 1e-300), value = sqrt(-2 ln u1) * exp(2 pi i u2); on the kx = 0
line |ky| keys the draw and ky < 0 takes the conjugate.  Commands apply in the
reference's order: density, then momentum, then order parameter
(src/project.h:92-116).
"""
from __future__ import annotations

import math
from typing import Dict, List, Tuple

import numpy as np

_M64 = (1 << 64) - 1


def _splitmix64(x: np.ndarray) -> np.ndarray:
    x = (x + np.uint64(0x9E3779B97F4A7C15)) & np.uint64(_M64)
    x = ((x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & np.uint64(_M64)
    x = ((x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & np.uint64(_M64)
    return x ^ (x >> np.uint64(31))


def _uniform(seed: int, channel: int, gx: np.ndarray, ky: np.ndarray, draw: int) -> np.ndarray:
    key = np.uint64(seed & 0xFFFFFFFF)
    key = key ^ (np.uint64(channel & 0xFFFFFFFF) << np.uint64(48))
    k = np.full(gx.shape, key, dtype=np.uint64)
    k ^= (gx.astype(np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)) << np.uint64(32)
    k ^= (ky.astype(np.int64).astype(np.uint64) & np.uint64(0xFFFFFFFF)) << np.uint64(8)
    k ^= np.uint64(draw & 0xFFFFFFFF)
    r = _splitmix64(k)
    return (r >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


class _Grid:
    def __init__(self, active: Tuple[int, int], grid: Tuple[int, int], length: Tuple[float, float]):
        self.nax, self.nay = active
        self.nx, self.ny = grid
        self.hx = self.nx // 2 + 1
        gx = np.arange(self.hx)
        gy = np.arange(self.ny)
        sgy = np.where(gy <= self.ny // 2, gy, gy - self.ny)
        self.gx = np.broadcast_to(gx[None, :], (self.ny, self.hx))
        self.sgy = np.broadcast_to(sgy[:, None], (self.ny, self.hx))
        kx = 2.0 * math.pi * self.gx / length[0]
        ky = 2.0 * math.pi * self.sgy / length[1]
        self.k2 = kx * kx + ky * ky
        self.active = (self.gx < self.nax // 2) & (np.abs(self.sgy) < self.nay // 2)
        self.grid_size = float(self.nx) * float(self.ny)
        self.volume = length[0] * length[1]

    def gaussian_modes(self, seed: int, channel: int) -> np.ndarray:
        phase_ky = np.where(self.gx == 0, np.abs(self.sgy), self.sgy)
        u1 = np.maximum(_uniform(seed, channel, self.gx, phase_ky, 0), 1.0e-300)
        u2 = _uniform(seed, channel, self.gx, phase_ky, 1)
        r = np.sqrt(-2.0 * np.log(u1))
        th = 2.0 * math.pi * u2
        v = r * np.cos(th) + 1j * (r * np.sin(th))
        return np.where((self.gx == 0) & (self.sgy < 0), np.conj(v), v)


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
            targets = list(range(n)) if t[2] == "all" else [int(t[2])]
            for a in targets:
                psi.append((a, t[3], _kv(t[4:])))
    return dens, mom, psi


def initial_state(cfg, script_text: str) -> np.ndarray:
    """State from the `set` lines of a script; cfg is a shhd_b200.Config (grid, length, N)."""
    g = _Grid((cfg.active_nx, cfg.active_ny), (cfg.nx, cfg.ny), (cfg.lx, cfg.ly))
    n = cfg.num_order_parameters
    u = np.zeros((n + 3, g.ny, g.hx), dtype=np.complex128)
    dens, mom, psi = _set_commands(cfg, script_text)
    act = g.active
    for style, kv in dens:
        rho = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            rho[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "equilibrium/gaussian":
            kbt, rho0, cT, seed = float(kv["kBT"]), float(kv.get("rho0", 1.0)), float(kv["cT"]), int(kv.get("seed", 0))
            rho[0, 0] = rho0 * g.grid_size
            if kbt != 0.0:
                cell = g.volume / g.grid_size
                sigma = math.sqrt(kbt * g.grid_size * rho0 / (2.0 * (cT * cT) * cell))
                modes = sigma * g.gaussian_modes(seed, 0)
                rho = np.where(act & (g.k2 != 0.0), modes, rho)
        else:
            raise NotImplementedError(f"set density {style}")
        u[0] = rho
    for d, style, kv in mom:
        f = n + 1 + d
        m = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            m[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "equilibrium/gaussian/compressible":
            kbt, seed = float(kv["kBT"]), int(kv.get("seed", 0))
            if kbt != 0.0:
                rho0 = u[0, 0, 0].real / g.grid_size
                if rho0 <= 0.0:
                    raise ValueError("set momentum equilibrium/gaussian/compressible requires positive reference density.")
                cell = g.volume / g.grid_size
                sigma = math.sqrt(kbt * g.grid_size * rho0 / (2.0 * cell))
                m = np.where(act & (g.k2 != 0.0), sigma * g.gaussian_modes(seed, d), 0.0)
        else:
            raise NotImplementedError(f"set momentum {style}")
        u[f] = m
    for a, style, kv in psi:
        f = 1 + a
        p = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if style == "uniform":
            p[0, 0] = float(kv["value"]) * g.grid_size
        elif style == "equilibrium/gaussian":
            kbt, seed, psi0 = float(kv["kBT"]), int(kv.get("seed", 0)), float(kv.get("psi0", 0.0))
            k0, k2c, k4 = float(kv.get("k0", 0.0)), float(kv.get("k2", 0.0)), float(kv.get("k4", 0.0))
            p[0, 0] = psi0 * g.grid_size
            if kbt != 0.0:
                coef = k0 + k2c * g.k2 + k4 * g.k2 * g.k2
                use = act & (g.k2 != 0.0)
                if np.any(coef[use] <= 0.0):
                    raise ValueError("set order_parameter equilibrium/gaussian requires positive linear chemical-potential "
                                     "coefficient for every active nonzero mode.")
                cell = g.volume / g.grid_size
                with np.errstate(divide="ignore", invalid="ignore"):
                    sigma = np.sqrt(kbt * g.grid_size / (2.0 * coef * cell))
                p = np.where(use, sigma * g.gaussian_modes(seed, a), p)
        else:
            raise NotImplementedError(f"set order_parameter {style}")
        u[f] = p
    return u


def field_generators(cfg, script_text: str) -> List[Tuple[int, int, int, float, float, float, float, float]]:
    """One (field, seed, channel, mean, s0, c0, c2, c4) per field: the state `initial_state` builds,
    as sigma(k)^2 = s0 / (c0 + c2 k^2 + c4 k^4) per active mode k != 0 and `mean` at k = 0.

    Every `set` command rewrites its whole field, so the last command on a field decides it; the
    momentum styles read the reference density the density commands left (src/project.h:92-116).
    """
    n = cfg.num_order_parameters
    ng = float(cfg.nx) * float(cfg.ny)
    cell = cfg.lx * cfg.ly / ng
    gens = {f: (f, 0, 0, 0.0, 0.0, 1.0, 0.0, 0.0) for f in range(n + 3)}
    dens, mom, psi = _set_commands(cfg, script_text)
    for style, kv in dens:
        if style == "uniform":
            gens[0] = (0, 0, 0, float(kv["value"]) * ng, 0.0, 1.0, 0.0, 0.0)
        elif style == "equilibrium/gaussian":
            kbt, rho0, cT, seed = float(kv["kBT"]), float(kv.get("rho0", 1.0)), float(kv["cT"]), int(kv.get("seed", 0))
            s0 = kbt * ng * rho0 / (2.0 * (cT * cT) * cell) if kbt != 0.0 else 0.0
            gens[0] = (0, seed, 0, rho0 * ng, s0, 1.0, 0.0, 0.0)
        else:
            raise NotImplementedError(f"set density {style}")
    rho0 = gens[0][3] / ng
    for d, style, kv in mom:
        f = n + 1 + d
        if style == "uniform":
            gens[f] = (f, 0, d, float(kv["value"]) * ng, 0.0, 1.0, 0.0, 0.0)
        elif style == "equilibrium/gaussian/compressible":
            kbt, seed = float(kv["kBT"]), int(kv.get("seed", 0))
            s0 = 0.0
            if kbt != 0.0:
                if rho0 <= 0.0:
                    raise ValueError("set momentum equilibrium/gaussian/compressible requires positive reference density.")
                s0 = kbt * ng * rho0 / (2.0 * cell)
            gens[f] = (f, seed, d, 0.0, s0, 1.0, 0.0, 0.0)
        else:
            raise NotImplementedError(f"set momentum {style}")
    for a, style, kv in psi:
        f = 1 + a
        if style == "uniform":
            gens[f] = (f, 0, a, float(kv["value"]) * ng, 0.0, 1.0, 0.0, 0.0)
        elif style == "equilibrium/gaussian":
            kbt, seed, psi0 = float(kv["kBT"]), int(kv.get("seed", 0)), float(kv.get("psi0", 0.0))
            k0, k2c, k4 = float(kv.get("k0", 0.0)), float(kv.get("k2", 0.0)), float(kv.get("k4", 0.0))
            s0 = kbt * ng / (2.0 * cell) if kbt != 0.0 else 0.0
            gens[f] = (f, seed, a, psi0 * ng, s0, k0, k2c, k4)
        else:
            raise NotImplementedError(f"set order_parameter {style}")
    return [gens[f] for f in range(n + 3)]


def initial_state_device(engine, script_text: str, member: int = 0) -> None:
    """Write the state of a script's `set` lines into one member of `engine`, generated on the device.

    The draws are those of `initial_state`; no state crosses PCIe (one kernel per field).
    """
    for f, seed, channel, mean, s0, c0, c2, c4 in field_generators(engine.cfg, script_text):
        engine.set_gaussian_field(member, f, seed, channel, mean, s0, c0, c2, c4)
