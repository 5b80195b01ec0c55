"""FP64 CPU restatement of the reference solver's per-step hot path (numpy).

TEST INFRASTRUCTURE ONLY.  This module is the oracle: the parity tests, the
smoke check and the CPU-baseline leg of bench.py call it as the checker.  The
product (the CUDA library and its host code) never imports it.

What it restates, with the reference file:line each part follows (paths are
relative to the reference project):

  * layout, k-vectors, mask .......... src/domain.cc:21-30,139-149,
                                       src/spectral_mask.cc:7-58, src/state.cc:22-38
  * 2-D R2C / C2R transforms ........ src/fourier_transform.h:39-51 (forward
                                       unscaled, backward scaled by 1/(Nx*Ny))
  * physical fields, v = j/rho ...... src/fcalculator_workspace.cc:41-145
  * rho_det ......................... src/fcalculator.cc:60-84
  * psi_det + linear/physical terms . src/fcalculator.cc:86-108,152-274
  * j_det, pressure, viscosity,
    advection ....................... src/fcalculator.cc:110-150,276-494
  * sine / gradient forces .......... src/fcalculator.cc:702-840
  * psi_sto / j_sto (noise -> RHS) .. src/fcalculator.cc:496-700
  * real-symmetry projection ........ src/time_integrator.h:70-109
  * Euler / SRK3 stage updates ...... src/time_integrator_euler_*.h,
                                       src/time_integrator_srk3_*.h

Free-energy plugin styles (``PLUGINS``) are the engine's own compile-time styles
(its csrc/free_energy_plugins.h); the reference has only the registry seam they
plug into (src/model_free_energy_registry.h:65-85), so their physical chemical
potentials and densities are restated here from the engine's definitions.

State layout is the reference's: complex128 array [field, gy, gx] with
gx in [0, Nx/2] (Nx, Ny = compute grid), field order rho, psi_0..psi_{N-1},
jx, jy.  Noise can come from (a) the reference's own draws replayed as
stochastic-RHS arrays ("external"), or (b) the counter-based Philox4x32-10
scheme the CUDA path uses ("philox"), restated in ``philox_normals``.
"""
from __future__ import annotations

import dataclasses
import math
import re
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

SQRT2 = 1.41421356237309504880
SQRT3 = 1.73205080756887729352
# time_integrator_srk3_compressible.h:10-21
BETA = ((2.0 * SQRT2 + SQRT3) / 5.0, (-4.0 * SQRT2 + 3.0 * SQRT3) / 5.0, (SQRT2 - 2.0 * SQRT3) / 10.0)
STAGE_WEIGHTS = ((0.0, 1.0), (3.0 / 4.0, 1.0 / 4.0), (1.0 / 3.0, 2.0 / 3.0))


# --------------------------------------------------------------------------
# configuration (the hot-path subset of the input-script grammar,
# src/param_parser.cc:42-163,165-339,581-639,641-769)
# --------------------------------------------------------------------------
@dataclasses.dataclass
class SineForce:
    target: str  # "momentum" | "order_parameter"
    component: int
    axis: int
    nk: int
    amplitude: float


@dataclasses.dataclass
class GradientForce:
    component: int
    direction: int
    amplitude: float


# Free-energy plugin styles: name -> (mu(a, psi, par), density(psi, par), parameter keys); psi the
# list of order-parameter fields, par {key without "[]": list of values}
def _coupled_phi4_mu(a, psi, par):
    others = sum(psi[b] * psi[b] for b in range(len(psi)) if b != a) if len(psi) > 1 else 0.0 * psi[a]
    return par["u"][a] * psi[a] * psi[a] * psi[a] + par["g"][0] * psi[a] * others


def _coupled_phi4_density(psi, par):
    q = [p * p for p in psi]
    s2, s4 = sum(q), sum(x * x for x in q)
    return sum(0.25 * par["u"][b] * q[b] * q[b] for b in range(len(psi))) + 0.25 * par["g"][0] * (s2 * s2 - s4)


def _phi6_mu(a, psi, par):
    q = psi[a] * psi[a]
    return psi[a] * q * (par["u"][a] + par["w"][a] * q)


def _phi6_density(psi, par):
    return sum((p * p) ** 2 * (0.25 * par["u"][b] + par["w"][b] * (p * p) / 6.0) for b, p in enumerate(psi))


PLUGINS = {
    "coupled_phi4": (_coupled_phi4_mu, _coupled_phi4_density, ("u[]", "g")),
    "phi6": (_phi6_mu, _phi6_density, ("u[]", "w[]")),
}


@dataclasses.dataclass
class Config:
    active: Tuple[int, int] = (128, 128)
    length: Tuple[float, float] = (2.0 * math.pi, 2.0 * math.pi)
    dealias: str = "none"
    num_order_parameters: int = 0
    dt: float = 0.005
    time_evolution: str = "srk3/compressible"
    cT: float = 0.0
    has_thermo: bool = False
    free_energy: str = "none"  # none | phi4 | quadratic | a PLUGINS name
    plugin_par: dict = dataclasses.field(default_factory=dict)
    phi4_a: List[float] = dataclasses.field(default_factory=list)
    phi4_b: List[float] = dataclasses.field(default_factory=list)
    phi4_u: List[float] = dataclasses.field(default_factory=list)
    quad_a: List[float] = dataclasses.field(default_factory=list)
    eta: float = 0.0
    zeta: float = 0.0
    mobility: List[float] = dataclasses.field(default_factory=list)
    momentum_advection: bool = False
    order_parameter_advection: bool = False
    noise_momentum: bool = False
    noise_order_parameter: bool = False
    noise_seed: int = 12345
    kBT: float = 1.0
    chi: float = 1.0
    sine_forces: List[SineForce] = dataclasses.field(default_factory=list)
    gradient_forces: List[GradientForce] = dataclasses.field(default_factory=list)

    @property
    def grid(self) -> Tuple[int, int]:
        def comp(n: int) -> int:
            if self.dealias == "none":
                return n
            if self.dealias == "3/2":
                return 3 * n // 2
            return 2 * n
        return comp(self.active[0]), comp(self.active[1])

    @property
    def mode(self) -> str:
        return self.time_evolution.split("/")[1]

    @property
    def integrator(self) -> str:
        return self.time_evolution.split("/")[0]

    @property
    def nfields(self) -> int:
        return self.num_order_parameters + 3

    def mu_k0(self, a: int) -> float:
        if self.free_energy == "phi4" or self.free_energy in PLUGINS:
            return self.phi4_a[a]
        if self.free_energy == "quadratic":
            return self.quad_a[a]
        return 0.0

    def mu_k2(self, a: int) -> float:
        return self.phi4_b[a] if (self.free_energy == "phi4" or self.free_energy in PLUGINS) else 0.0

    def has_physical_mu(self) -> bool:
        return self.free_energy in PLUGINS or (self.free_energy == "phi4" and any(u != 0.0 for u in self.phi4_u))

    def physical_mu(self, a: int, psi) -> np.ndarray:
        """Physical chemical potential of order parameter a from the physical fields psi."""
        if self.free_energy in PLUGINS:
            return PLUGINS[self.free_energy][0](a, psi, self.plugin_par)
        return self.phi4_u[a] * psi[a] * psi[a] * psi[a]

    def physical_density(self, psi) -> np.ndarray:
        """Free-energy density of the physical part."""
        if self.free_energy in PLUGINS:
            return PLUGINS[self.free_energy][1](psi, self.plugin_par)
        return sum(0.25 * self.phi4_u[a] * p ** 4 for a, p in enumerate(psi))


def parse_script(text: str) -> Config:
    """Parse the hot-path commands of a reference input script.

    Follows src/param_parser.cc (execute_command 42-163, model 165-284,
    fix 287-339 / 551-769).  Initial-condition, measure, thermo, restart and
    run lines are accepted and ignored here (they do not shape the step).
    """
    c = Config()
    n_op = 0
    for raw in text.splitlines():
        t = raw.split("#", 1)[0].split()
        if not t:
            continue
        cmd = t[0]
        if cmd == "grid":
            c.active = (int(t[1]), int(t[2]))
        elif cmd == "length":
            c.length = (float(t[1]), float(t[2]))
        elif cmd == "dealias":
            r = t[1]
            c.dealias = {"none": "none", "off": "none", "three_halves": "3/2", "3/2": "3/2", "two": "2", "2": "2"}[r]
        elif cmd in ("order_parameters", "order_parameter"):
            n_op = int(t[1])
            c.num_order_parameters = n_op
        elif cmd == "timestep":
            c.dt = float(t[1])
        elif cmd == "time_evolution":
            c.time_evolution = t[1]
        elif cmd == "model":
            kv = list(zip(t[3::2], t[4::2]))
            if t[1] == "thermo":
                c.has_thermo = True
                for k, v in kv:
                    if k in ("cT", "sound_speed"):
                        c.cT = float(v)
            elif t[1] == "free_energy":
                c.free_energy = t[2]
                c.phi4_a = [0.0] * n_op
                c.phi4_b = [0.0] * n_op
                c.phi4_u = [0.0] * n_op
                c.quad_a = [0.0] * n_op
                if c.free_energy in PLUGINS:
                    c.plugin_par = {key.rstrip("[]"): [0.0] * max(n_op, 1) for key in PLUGINS[c.free_energy][2]}
                    for k, v in kv:
                        m = re.fullmatch(r"(\w+)\[(\d+)\]", k)
                        if m and m.group(1) in ("a", "b"):
                            (c.phi4_a if m.group(1) == "a" else c.phi4_b)[int(m.group(2))] = float(v)
                        elif m:
                            c.plugin_par[m.group(1)][int(m.group(2))] = float(v)
                        else:
                            c.plugin_par[k][0] = float(v)
                    continue
                for k, v in kv:
                    m = re.fullmatch(r"([abu])\[(\d+)\]", k)
                    if m:
                        arr = {"a": c.phi4_a if c.free_energy == "phi4" else c.quad_a, "b": c.phi4_b, "u": c.phi4_u}[m.group(1)]
                        arr[int(m.group(2))] = float(v)
            elif t[1] == "transport":
                c.mobility = [0.0] * n_op
                for k, v in kv:
                    if k in ("eta", "shear_viscosity"):
                        c.eta = float(v)
                    elif k in ("zeta", "bulk_viscosity"):
                        c.zeta = float(v)
                    else:
                        m = re.fullmatch(r"M\[(\d+),(\d+)\]", k)
                        if m and m.group(1) == m.group(2):
                            c.mobility[int(m.group(1))] = float(v)
        elif cmd == "fix":
            target = {"momentum": "momentum", "j": "momentum", "order_parameter": "order_parameter", "psi": "order_parameter", "all": "all"}[t[2]]
            kind, on = t[3], t[4] == "on"
            if kind == "nonlinear":
                if target in ("momentum", "all"):
                    c.momentum_advection = on
                if target in ("order_parameter", "all"):
                    c.order_parameter_advection = on and n_op > 0
            elif kind == "noise":
                for k, v in zip(t[5::2], t[6::2]):
                    if k == "seed":
                        c.noise_seed = int(v)
                    elif k in ("kBT", "temperature"):
                        c.kBT = float(v)
                    elif k in ("chi", "order_parameter_chi", "psi_chi"):
                        c.chi = float(v)
                if target in ("momentum", "all"):
                    c.noise_momentum = on
                if target in ("order_parameter", "all"):
                    c.noise_order_parameter = on and n_op > 0
                if c.mode == "quiescent":
                    c.noise_momentum = False
            elif kind == "force/sine" and on:
                kv = dict(zip(t[5::2], t[6::2]))
                xy = {"x": 0, "0": 0, "y": 1, "1": 1}
                comp = xy[kv["component"]] if target == "momentum" else int(kv["component"])
                c.sine_forces.append(SineForce(target, comp, xy[kv["axis"]], int(kv["nk"]), float(kv["amplitude"])))
            elif kind == "force/gradient" and on:
                kv = dict(zip(t[5::2], t[6::2]))
                xy = {"x": 0, "0": 0, "y": 1, "1": 1}
                c.gradient_forces.append(GradientForce(int(kv["component"]), xy[kv["direction"]], float(kv["amplitude"])))
    if not c.mobility:
        c.mobility = [0.0] * n_op
    return c


# --------------------------------------------------------------------------
# spectral geometry (src/domain.cc:139-149, src/spectral_mask.cc:7-52)
# --------------------------------------------------------------------------
class Geometry:
    def __init__(self, cfg: Config):
        self.cfg = cfg
        self.nx, self.ny = cfg.grid
        self.nax, self.nay = cfg.active
        self.hx = self.nx // 2 + 1
        gx = np.arange(self.hx)
        gy = np.arange(self.ny)
        sgy = np.where(gy <= self.ny // 2, gy, gy - self.ny)
        self.gx = gx[None, :].repeat(self.ny, 0)
        self.gy = gy[:, None].repeat(self.hx, 1)
        self.sgy = sgy[:, None].repeat(self.hx, 1)
        self.kx = (2.0 * math.pi * gx / cfg.length[0])[None, :].repeat(self.ny, 0)
        self.ky = (2.0 * math.pi * sgy / cfg.length[1])[:, None].repeat(self.hx, 1)
        self.k2 = self.kx * self.kx + self.ky * self.ky
        self.active = (self.gx < self.nax // 2) & (np.abs(self.sgy) < self.nay // 2)
        self.grid_size = float(self.nx) * float(self.ny)
        self.volume = cfg.length[0] * cfg.length[1]

    def backward(self, f: np.ndarray) -> np.ndarray:
        """C2R with scale::full (fourier_transform.h:46-51)."""
        return np.fft.irfft2(f, s=(self.ny, self.nx), axes=(-2, -1))

    def forward(self, p: np.ndarray) -> np.ndarray:
        """R2C with scale::none (fourier_transform.h:39-44)."""
        return np.fft.rfft2(p, axes=(-2, -1))


# --------------------------------------------------------------------------
# Philox4x32-10 counter-based normals (the CUDA path's noise scheme)
# --------------------------------------------------------------------------
_PHILOX_M0 = np.uint64(0xD2511F53)
_PHILOX_M1 = np.uint64(0xCD9E8D57)
_PHILOX_W0 = 0x9E3779B9
_PHILOX_W1 = 0xBB67AE85
_MASK32 = np.uint64(0xFFFFFFFF)


def philox4x32_10(c0, c1, c2, c3, k0: int, k1: int):
    """Philox4x32 with 10 rounds (Salmon et al., SC'11), vectorised over counters."""
    c0 = np.asarray(c0, dtype=np.uint64) & _MASK32
    c1 = np.asarray(c1, dtype=np.uint64) & _MASK32
    c2 = np.asarray(c2, dtype=np.uint64) & _MASK32
    c3 = np.asarray(c3, dtype=np.uint64) & _MASK32
    c0, c1, c2, c3 = np.broadcast_arrays(c0, c1, c2, c3)
    k0 = int(k0) & 0xFFFFFFFF
    k1 = int(k1) & 0xFFFFFFFF
    for r in range(10):
        if r > 0:
            k0 = (k0 + _PHILOX_W0) & 0xFFFFFFFF
            k1 = (k1 + _PHILOX_W1) & 0xFFFFFFFF
        p0 = _PHILOX_M0 * c0
        p1 = _PHILOX_M1 * c2
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK32
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK32
        c0, c1, c2, c3 = hi1 ^ c1 ^ np.uint64(k0), lo1, hi0 ^ c3 ^ np.uint64(k1), lo0
    return c0, c1, c2, c3


def philox_normals(seed: int, member: int, step: int, stream: int, mode_id):
    """The two complex standard normals (draws a and b) of one noise component per mode id.

    counter = (mode_id, stream, step_lo, step_hi), key = (seed, member);
    draw a from words (w0, w1), draw b from (w2, w3); u = (w + 1/2) 2^-32;
    Box-Muller: r = sqrt(-2 ln u1), theta = 2 pi u2.
    """
    step = int(step)
    w0, w1, w2, w3 = philox4x32_10(mode_id, stream, step & 0xFFFFFFFF, (step >> 32) & 0xFFFFFFFF, seed, member)

    def bm(wr, wt):
        u1 = (wr.astype(np.float64) + 0.5) * 2.3283064365386963e-10
        u2 = (wt.astype(np.float64) + 0.5) * 2.3283064365386963e-10
        r = np.sqrt(-2.0 * np.log(u1))
        return r * np.cos(2.0 * math.pi * u2) + 1j * r * np.sin(2.0 * math.pi * u2)

    return bm(w0, w1), bm(w2, w3)


# stream ids: psi component alpha -> alpha; momentum stress draws xi_1..xi_3 -> 4096 + m
def psi_stream(alpha: int) -> int:
    return alpha


def j_stream(m: int) -> int:
    return 4096 + m


class PhysicalFields:
    """Inverse-transformed fields of one state, computed on first use.

    The velocity is built only when a term asks for it, as in
    fcalculator_workspace.cc:115-142, so the zero-density check fires in the
    same cases as the reference's.
    """

    def __init__(self, oracle: "Oracle", state: np.ndarray):
        self._o = oracle
        self._s = state
        self._cache: Dict[str, np.ndarray] = {}

    def __getitem__(self, key: str) -> np.ndarray:
        if key not in self._cache:
            self._cache[key] = self._make(key)
        return self._cache[key]

    def _make(self, key: str) -> np.ndarray:
        o, s = self._o, self._s
        g, n = o.geo, o.cfg.num_order_parameters
        if key == "psi":
            return g.backward(s[1:1 + n])
        if key == "rho":
            return g.backward(s[0])
        if key == "jx":
            return g.backward(s[n + 1])
        if key == "jy":
            return g.backward(s[n + 2])
        if key in ("vx", "vy"):
            if o.cfg.mode == "compressible":
                rho = self["rho"]
                if np.any(rho == 0.0):
                    raise RuntimeError("compressible velocity encountered zero density.")
                self._cache["vx"] = self["jx"] / rho
                self._cache["vy"] = self["jy"] / rho
            else:
                rho0 = o.reference_density(s)
                self._cache["vx"] = self["jx"] / rho0
                self._cache["vy"] = self["jy"] / rho0
            return self._cache[key]
        raise KeyError(key)


# --------------------------------------------------------------------------
# the right-hand side (src/fcalculator.cc)
# --------------------------------------------------------------------------
class Oracle:
    """FCalculator + TimeIntegrator restated over numpy arrays."""

    def __init__(self, cfg: Config, member: int = 0):
        self.cfg = cfg
        self.geo = Geometry(cfg)
        self.member = member
        self.rho0_cached: Optional[float] = None
        self.step_index = 0
        self.time = 0.0
        g = self.geo
        self.shape = (cfg.nfields, g.ny, g.hx)

    # --- helpers -----------------------------------------------------------
    def _mask(self, f: np.ndarray) -> np.ndarray:
        return np.where(self.geo.active, f, 0.0)

    def reference_density(self, state: np.ndarray) -> float:
        """fcalculator_workspace.cc:41-66 (cached after the first call)."""
        if self.rho0_cached is None:
            rho0 = state[0, 0, 0].real / self.geo.grid_size
            if rho0 == 0.0:
                raise RuntimeError("reference density must be nonzero.")
            self.rho0_cached = rho0
        return self.rho0_cached

    def physical_fields(self, state: np.ndarray) -> "PhysicalFields":
        """ensure_physical_fields (fcalculator_workspace.cc:68-145)."""
        return PhysicalFields(self, state)

    def rhs(self, state: np.ndarray) -> np.ndarray:
        """Deterministic RHS for every field, State field order."""
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        det = np.zeros(self.shape, dtype=np.complex128)
        phys: Optional[PhysicalFields] = None

        def need_phys():
            nonlocal phys
            if phys is None:
                phys = self.physical_fields(state)
            return phys

        kx, ky, k2 = g.kx, g.ky, g.k2
        act = g.active
        mi = -1j

        # rho_det (fcalculator.cc:60-84)
        if cfg.mode == "compressible":
            det[0] = np.where(act, mi * (kx * state[n + 1] + ky * state[n + 2]), 0.0)

        # psi_det (fcalculator.cc:86-108)
        for a in range(n):
            out = np.zeros((g.ny, g.hx), dtype=np.complex128)
            M = cfg.mobility[a]
            adv = cfg.order_parameter_advection
            if M == 0.0 and not adv:
                det[1 + a] = out
                continue
            if M != 0.0:
                k0c, k2c = cfg.mu_k0(a), cfg.mu_k2(a)
                if k0c != 0.0 or k2c != 0.0:
                    mu_hat = (k0c + k2c * k2 + 0.0 * k2 * k2) * state[1 + a]
                    jxf = -1j * (M * kx) * mu_hat
                    jyf = -1j * (M * ky) * mu_hat
                    out += np.where(act, mi * (kx * jxf + ky * jyf), 0.0)
            if adv or cfg.has_physical_mu():
                p = need_phys()
                has_mu = M != 0.0 and cfg.has_physical_mu()
                if has_mu:
                    mu = cfg.physical_mu(a, p["psi"])
                    mu_hat = g.forward(mu)
                    jxf = -1j * (M * kx) * mu_hat
                    jyf = -1j * (M * ky) * mu_hat
                    out += np.where(act, mi * (kx * jxf + ky * jyf), 0.0)
                if adv:
                    fx = g.forward(p["psi"][a] * p["vx"])
                    fy = g.forward(p["psi"][a] * p["vy"])
                    out += np.where(act, mi * (kx * fx + ky * fy), 0.0)
            # sine force (fcalculator.cc:741-774)
            for f in cfg.sine_forces:
                if f.target == "order_parameter" and f.component == a:
                    out += self._sine_source(f)
            # gradient force (fcalculator.cc:776-840)
            grads = [f for f in cfg.gradient_forces if f.component == a]
            if grads:
                if cfg.mode == "quiescent":
                    raise RuntimeError("force/gradient cannot be used in quiescent mode.")
                if cfg.mode == "incompressible":
                    rho0 = self.reference_density(state)
                    for f in grads:
                        mom = state[n + 1] if f.direction == 0 else state[n + 2]
                        out += np.where(act, -f.amplitude * mom / rho0, 0.0)
                else:
                    p = need_phys()
                    src = np.zeros((g.ny, g.nx))
                    for f in grads:
                        src += -f.amplitude * (p["vx"] if f.direction == 0 else p["vy"])
                    out += np.where(act, g.forward(src), 0.0)
            det[1 + a] = out

        # j_det (fcalculator.cc:110-150)
        if cfg.mode != "quiescent":
            ox = np.zeros((g.ny, g.hx), dtype=np.complex128)
            oy = np.zeros((g.ny, g.hx), dtype=np.complex128)
            pc = cfg.cT * cfg.cT
            eta, zeta = cfg.eta, cfg.zeta
            has_visc = eta != 0.0 or zeta != 0.0
            adv = cfg.momentum_advection
            if pc != 0.0 or has_visc or adv:
                if pc != 0.0:  # add_linear_pressure_term 276-300
                    ph = pc * state[0]
                    ox += np.where(act, -1j * kx * ph, 0.0)
                    oy += np.where(act, -1j * ky * ph, 0.0)
                if has_visc and cfg.mode == "incompressible" and eta != 0.0:  # 302-341
                    rho0 = self.reference_density(state)
                    vx = state[n + 1] / rho0
                    vy = state[n + 2] / rho0
                    pxx = -1j * eta * (2.0 * kx * vx)
                    pxy = -1j * eta * (ky * vx + kx * vy)
                    pyy = -1j * eta * (2.0 * ky * vy)
                    ox += np.where(act, mi * (kx * pxx + ky * pxy), 0.0)
                    oy += np.where(act, mi * (kx * pxy + ky * pyy), 0.0)
                if has_visc and cfg.mode == "compressible":  # 343-398
                    p = need_phys()
                    vx = g.forward(p["vx"])
                    vy = g.forward(p["vy"])
                    kv = kx * vx + ky * vy
                    pxx = -1j * (2.0 * eta * kx * vx - (eta - zeta) * kv)
                    pxy = -1j * eta * (ky * vx + kx * vy)
                    pyy = -1j * (2.0 * eta * ky * vy - (eta - zeta) * kv)
                    ox += np.where(act, mi * (kx * pxx + ky * pxy), 0.0)
                    oy += np.where(act, mi * (kx * pxy + ky * pyy), 0.0)
                if adv:  # add_momentum_physical_terms 400-494
                    p = need_phys()
                    pxx = g.forward(p["jx"] * p["vx"])
                    pxy = g.forward(p["jx"] * p["vy"])
                    pyy = g.forward(p["jy"] * p["vy"])
                    ox += np.where(act, mi * (kx * pxx + ky * pxy), 0.0)
                    oy += np.where(act, mi * (kx * pxy + ky * pyy), 0.0)
                for f in cfg.sine_forces:  # 702-739
                    if f.target == "momentum":
                        s = self._sine_source(f)
                        if f.component == 0:
                            ox += s
                        else:
                            oy += s
            det[n + 1] = ox
            det[n + 2] = oy
        return det

    def _sine_source(self, f: SineForce) -> np.ndarray:
        g = self.geo
        src = np.zeros((g.ny, g.hx), dtype=np.complex128)
        pos = complex(0.0, -0.5 * f.amplitude * g.grid_size)
        gxp = f.nk if f.axis == 0 else 0
        gyp = 0 if f.axis == 0 else f.nk
        gyn = (g.ny - f.nk) % g.ny
        if g.active[gyp, gxp]:
            src[gyp, gxp] += pos
        if f.axis == 1 and g.active[gyn, 0]:
            src[gyn, 0] += pos.conjugate()
        return src

    # --- noise: normals -> stochastic RHS (fcalculator.cc:496-700) ---------
    def noise_from_normals(self, xi_psi: Sequence[np.ndarray], xi_j: Sequence[np.ndarray]) -> np.ndarray:
        """Stochastic RHS from complex normals laid out like a spectral field.

        ``xi_psi[a]`` and ``xi_j[m]`` (m = 0,1,2) hold one complex normal per
        (gy, gx).  On the kx = 0 line only 0 < gy < Ny/2 is read; the
        conjugate partner is filled as the reference does.
        """
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        sto = np.zeros(self.shape, dtype=np.complex128)
        use = g.active & (g.k2 != 0.0)
        line = use & (g.gx == 0) & (g.gy < (g.ny - g.gy) % g.ny)
        bulk = use & (g.gx != 0)
        conj_rows = (g.ny - np.arange(g.ny)) % g.ny
        kx, ky, k2 = g.kx, g.ky, g.k2
        if cfg.noise_order_parameter:
            kbt = cfg.kBT * cfg.chi
            pref = 2.0 * kbt * g.grid_size * g.grid_size / g.volume
            for a in range(n):
                M = cfg.mobility[a]
                if M == 0.0 or kbt == 0.0:
                    continue
                xi = xi_psi[a]
                sig = np.sqrt(0.5 * pref * M * k2)
                with np.errstate(divide="ignore", invalid="ignore"):
                    fx = np.where(bulk, 1j * (kx / k2) * sig * xi, 0.0)
                    fy = 1j * (ky / k2) * sig * xi
                val = -1j * (kx * fx + ky * fy)
                out = np.where(bulk, val, 0.0)
                linev = np.where(line, -1j * (0.0 * 0.0 + ky * fy), 0.0)
                out[:, 0] += linev[:, 0]
                out[conj_rows, 0] += np.conj(linev[:, 0])
                sto[1 + a] = out
        if cfg.noise_momentum and cfg.mode != "quiescent":
            kbt = cfg.kBT
            eta, zeta = cfg.eta, cfg.zeta
            if kbt != 0.0 and (eta != 0.0 or zeta != 0.0):
                pref = 2.0 * kbt * g.grid_size * g.grid_size / g.volume
                s = math.sqrt(0.5 * pref)
                se, sz = math.sqrt(eta), math.sqrt(zeta)
                x1, x2, x3 = xi_j
                pxx = -s * (sz * x1 + se * x2)
                pyy = -s * (sz * x1 - se * x2)
                pxy = -s * se * x3
                vx = -1j * (kx * pxx + ky * pxy)
                vy = -1j * (kx * pxy + ky * pyy)
                ox = np.where(bulk, vx, 0.0)
                oy = np.where(bulk, vy, 0.0)
                lx = np.where(line, vx, 0.0)
                ly = np.where(line, vy, 0.0)
                ox[:, 0] += lx[:, 0]
                oy[:, 0] += ly[:, 0]
                ox[conj_rows, 0] += np.conj(lx[:, 0])
                oy[conj_rows, 0] += np.conj(ly[:, 0])
                sto[n + 1] = ox
                sto[n + 2] = oy
        return sto

    def mode_ids(self) -> np.ndarray:
        """Philox mode id per (gy, gx): gx * Nay + (ky mod Nay), |ky| on kx = 0."""
        g = self.geo
        ky = np.where(g.gx == 0, np.abs(g.sgy), g.sgy)
        return (g.gx.astype(np.int64) * g.nay + np.mod(ky, g.nay)).astype(np.uint64)

    def philox_noise(self, step: int):
        """(sto_a, sto_b) of one step from the Philox scheme of the CUDA path."""
        cfg = self.cfg
        ids = self.mode_ids()
        xp = [philox_normals(cfg.noise_seed, self.member, step, psi_stream(a), ids) for a in range(cfg.num_order_parameters)]
        xj = [philox_normals(cfg.noise_seed, self.member, step, j_stream(m), ids) for m in range(3)]
        sa = self.noise_from_normals([x[0] for x in xp], [x[0] for x in xj])
        sb = self.noise_from_normals([x[1] for x in xp], [x[1] for x in xj])
        return sa, sb

    # --- symmetry (time_integrator.h:70-109) --------------------------------
    def enforce_real_symmetry(self, u: np.ndarray) -> np.ndarray:
        g = self.geo
        u = np.where(g.active[None], u, 0.0)
        ny = g.ny
        for gy in range(ny):
            if not g.active[gy, 0]:
                continue
            c = (ny - gy) % ny
            if c == gy:
                u[:, gy, 0] = u[:, gy, 0].real + 0j
                continue
            if gy > c:
                continue
            a = u[:, gy, 0].copy()
            b = u[:, c, 0].copy()
            p = 0.5 * (a + np.conj(b))
            u[:, gy, 0] = p
            u[:, c, 0] = np.conj(p)
        return u

    # --- integrators -------------------------------------------------------
    def _evolved(self) -> List[int]:
        n = self.cfg.num_order_parameters
        if self.cfg.mode == "compressible":
            return list(range(n + 3))
        return list(range(1, n + 1))

    def _stage(self, cur, base, sto, wb, wc):
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        dt = cfg.dt
        sdt = math.sqrt(dt)
        det = self.rhs(cur)
        act = g.active
        nxt = cur.copy()
        for f in self._evolved():
            nxt[f] = np.where(act, wb * base[f] + wc * (cur[f] + dt * det[f] + sdt * sto[f]), cur[f])
        if cfg.mode == "incompressible":
            ix = dt * det[n + 1] + sdt * sto[n + 1]
            iy = dt * det[n + 2] + sdt * sto[n + 2]
            with np.errstate(divide="ignore", invalid="ignore"):
                tr = -g.ky * ix + g.kx * iy
                px = np.where(g.k2 != 0.0, -g.ky * tr / g.k2, ix)
                py = np.where(g.k2 != 0.0, g.kx * tr / g.k2, iy)
            nxt[n + 1] = np.where(act, wb * base[n + 1] + wc * (cur[n + 1] + px), cur[n + 1])
            nxt[n + 2] = np.where(act, wb * base[n + 2] + wc * (cur[n + 2] + py), cur[n + 2])
        return self.enforce_real_symmetry(nxt)

    def step(self, u: np.ndarray, noise=None) -> np.ndarray:
        """Advance one step.

        noise: None (no noise), "philox", or a tuple of stochastic-RHS arrays
        (sto_a, sto_b) for SRK3 / (sto,) for Euler in State layout.
        """
        cfg = self.cfg
        noisy = cfg.noise_order_parameter or (cfg.noise_momentum and cfg.mode != "quiescent")
        if noise is None or not noisy:
            zero = np.zeros(self.shape, dtype=np.complex128)
            sa, sb = zero, zero
        elif isinstance(noise, str):
            sa, sb = self.philox_noise(self.step_index)
        else:
            sa = noise[0]
            sb = noise[1] if cfg.integrator == "srk3" else None
        if cfg.integrator == "euler":
            out = self._stage(u, u, sa, 0.0, 1.0)
        else:
            u1 = self._stage(u, u, sa + BETA[0] * sb, *STAGE_WEIGHTS[0])
            u2 = self._stage(u1, u, sa + BETA[1] * sb, *STAGE_WEIGHTS[1])
            out = self._stage(u2, u, sa + BETA[2] * sb, *STAGE_WEIGHTS[2])
        self.step_index += 1
        self.time += cfg.dt
        return out


    # --- momentum flux pi_xy and the Yokota-Green-Kubo accumulation --------
    def momentum_flux_xy(self, state: np.ndarray) -> np.ndarray:
        """Deterministic pi_xy of one RHS evaluation, as j_det records it in the flux
        buffer: viscous (fcalculator.cc:302-341 incompressible, 343-398 compressible)
        plus advection (fcalculator.cc:400-494); the pressure enters pi_xx, pi_yy only."""
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        act = g.active
        kx, ky = g.kx, g.ky
        out = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if cfg.mode == "quiescent":
            return out
        eta, zeta = cfg.eta, cfg.zeta
        has_visc = eta != 0.0 or zeta != 0.0
        if not (cfg.cT * cfg.cT != 0.0 or has_visc or cfg.momentum_advection):
            return out
        p = None
        if has_visc and cfg.mode == "incompressible" and eta != 0.0:
            rho0 = self.reference_density(state)
            out += np.where(act, -1j * eta * (ky * state[n + 1] / rho0 + kx * state[n + 2] / rho0), 0.0)
        if has_visc and cfg.mode == "compressible":
            p = self.physical_fields(state)
            vx, vy = g.forward(p["vx"]), g.forward(p["vy"])
            out += np.where(act, -1j * eta * (ky * vx + kx * vy), 0.0)
        if cfg.momentum_advection:
            p = p or self.physical_fields(state)
            out += np.where(act, g.forward(p["jx"] * p["vy"]), 0.0)
        return out

    def k0_flux(self, state: np.ndarray) -> Dict[str, float]:
        """Real part of the (0, 0) coefficient of the fluxes one RHS evaluation records
        (unnormalised): the gradient terms (viscous, chemical potential, projection) vanish at
        k = 0 and no noise is drawn there, so pi_xx = pi_yy = cT^2 rho(0) + sum jx vx | jy vy,
        pi_xy = sum jx vy (fcalculator.cc:110-150, 276-300, 400-494) and Jpsi[a] = sum psi_a v
        (fcalculator.cc:86-108, 189-274), each term where the reference evaluates it."""
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        out = {"pi_xx": 0.0, "pi_xy": 0.0, "pi_yy": 0.0}
        for a in range(n):
            out[f"Jpsi[{a}]_x"] = out[f"Jpsi[{a}]_y"] = 0.0
        p = self.physical_fields(state)
        if cfg.mode != "quiescent":
            if cfg.cT * cfg.cT != 0.0:
                out["pi_xx"] += cfg.cT * cfg.cT * state[0, 0, 0].real
                out["pi_yy"] += cfg.cT * cfg.cT * state[0, 0, 0].real
            if cfg.momentum_advection:
                out["pi_xx"] += float(np.sum(p["jx"] * p["vx"]))
                out["pi_xy"] += float(np.sum(p["jx"] * p["vy"]))
                out["pi_yy"] += float(np.sum(p["jy"] * p["vy"]))
        if cfg.order_parameter_advection:
            psi = p["psi"]
            for a in range(n):
                out[f"Jpsi[{a}]_x"] += float(np.sum(psi[a] * p["vx"]))
                out[f"Jpsi[{a}]_y"] += float(np.sum(psi[a] * p["vy"]))
        return out

    def step_with_k0_flux(self, u: np.ndarray, noise=None):
        """(next state, the step's k = 0 flux columns of the time-series measure): the stage
        fluxes weighted 1/6, 1/6, 2/3 (SRK3) or 1 (Euler), divided by the grid size
        (time_integrator_srk3_compressible.h:99-146, measure_time_series.cc:190-229)."""
        cfg = self.cfg
        if cfg.integrator == "euler":
            stages, weights = [u], [1.0]
            out = self.step(u, noise)
        else:
            sa, sb = noise if noise is not None else (np.zeros(self.shape, complex),) * 2
            u1 = self._stage(u, u, sa + BETA[0] * sb, *STAGE_WEIGHTS[0])
            u2 = self._stage(u1, u, sa + BETA[1] * sb, *STAGE_WEIGHTS[1])
            out = self._stage(u2, u, sa + BETA[2] * sb, *STAGE_WEIGHTS[2])
            self.step_index += 1
            self.time += cfg.dt
            stages, weights = [u, u1, u2], [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]
        acc: Dict[str, float] = {}
        for w, st in zip(weights, stages):
            for k, v in self.k0_flux(st).items():
                acc[k] = acc.get(k, 0.0) + w * v
        return out, {k: v / self.geo.grid_size for k, v in acc.items()}

    def _mu_coefficients(self, a: int) -> Tuple[float, float, float]:
        cfg = self.cfg
        if cfg.free_energy == "phi4":
            return cfg.phi4_a[a], cfg.phi4_b[a], 0.0
        if cfg.free_energy == "quadratic":
            return cfg.quad_a[a], 0.0, 0.0
        return 0.0, 0.0, 0.0

    def flux_fields(self, state: np.ndarray) -> Dict[str, np.ndarray]:
        """Every flux one deterministic RHS evaluation records in the flux buffer, per mode:
        psi_det's -i M k mu (linear and physical chemical potential) and psi v (fcalculator.cc:86-274),
        j_det's linear pressure, viscous and advective stresses (fcalculator.cc:110-494), each where
        the reference evaluates it.  Keys pi_xx, pi_xy, pi_yy, Jpsi[a]_x, Jpsi[a]_y."""
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        act = g.active
        kx, ky, k2 = g.kx, g.ky, g.k2
        zero = lambda: np.zeros((g.ny, g.hx), dtype=np.complex128)  # noqa: E731
        out = {"pi_xx": zero(), "pi_xy": zero(), "pi_yy": zero()}
        for a in range(n):
            out[f"Jpsi[{a}]_x"], out[f"Jpsi[{a}]_y"] = zero(), zero()
        p = self.physical_fields(state)
        has_phys = cfg.has_physical_mu()
        for a in range(n):
            M = cfg.mobility[a]
            adv = cfg.order_parameter_advection
            if M == 0.0 and not adv:
                continue
            fx, fy = out[f"Jpsi[{a}]_x"], out[f"Jpsi[{a}]_y"]
            c0, c2, c4 = self._mu_coefficients(a)
            if M != 0.0 and (c0 != 0.0 or c2 != 0.0 or c4 != 0.0):
                mu = (c0 + c2 * k2 + c4 * k2 * k2) * state[1 + a]
                fx += np.where(act, -1j * (M * kx) * mu, 0.0)
                fy += np.where(act, -1j * (M * ky) * mu, 0.0)
            if adv or has_phys:
                if M != 0.0 and has_phys:
                    mu_p = g.forward(cfg.physical_mu(a, p["psi"]))
                    fx += np.where(act, -1j * (M * kx) * mu_p, 0.0)
                    fy += np.where(act, -1j * (M * ky) * mu_p, 0.0)
                if adv:
                    fx += np.where(act, g.forward(p["psi"][a] * p["vx"]), 0.0)
                    fy += np.where(act, g.forward(p["psi"][a] * p["vy"]), 0.0)
        if cfg.mode != "quiescent":
            eta, zeta = cfg.eta, cfg.zeta
            has_lp = cfg.cT * cfg.cT != 0.0
            has_visc = eta != 0.0 or zeta != 0.0
            if has_lp or has_visc or cfg.momentum_advection:
                xx, xy, yy = out["pi_xx"], out["pi_xy"], out["pi_yy"]
                if has_lp:
                    pr = cfg.cT * cfg.cT * state[0]
                    xx += np.where(act, pr, 0.0)
                    yy += np.where(act, pr, 0.0)
                if has_visc and cfg.mode == "incompressible" and eta != 0.0:
                    rho0 = self.reference_density(state)
                    vx, vy = state[n + 1] / rho0, state[n + 2] / rho0
                    xx += np.where(act, -1j * eta * (2.0 * kx * vx), 0.0)
                    xy += np.where(act, -1j * eta * (ky * vx + kx * vy), 0.0)
                    yy += np.where(act, -1j * eta * (2.0 * ky * vy), 0.0)
                if has_visc and cfg.mode == "compressible":
                    vx, vy = g.forward(p["vx"]), g.forward(p["vy"])
                    kv = kx * vx + ky * vy
                    xx += np.where(act, -1j * (2.0 * eta * kx * vx - (eta - zeta) * kv), 0.0)
                    xy += np.where(act, -1j * eta * (ky * vx + kx * vy), 0.0)
                    yy += np.where(act, -1j * (2.0 * eta * ky * vy - (eta - zeta) * kv), 0.0)
                if cfg.momentum_advection:
                    xx += np.where(act, g.forward(p["jx"] * p["vx"]), 0.0)
                    xy += np.where(act, g.forward(p["jx"] * p["vy"]), 0.0)
                    yy += np.where(act, g.forward(p["jy"] * p["vy"]), 0.0)
        return out

    def noise_flux_fields(self, xi_psi: Sequence[np.ndarray], xi_j: Sequence[np.ndarray]) -> Dict[str, np.ndarray]:
        """Fluxes psi_sto and j_sto record for one draw (fcalculator.cc:496-700): psi i k / k^2 sigma xi
        (x-component zero on the kx = 0 line), momentum -s (sqrt(zeta) xi1 +- sqrt(eta) xi2) on the
        diagonal and -s sqrt(eta) xi3 off it; on the kx = 0 line the drawn half and its conjugate."""
        cfg, g = self.cfg, self.geo
        n = cfg.num_order_parameters
        use = g.active & (g.k2 != 0.0)
        line = use & (g.gx == 0) & (g.gy < (g.ny - g.gy) % g.ny)
        bulk = use & (g.gx != 0)
        conj_rows = (g.ny - np.arange(g.ny)) % g.ny
        kx, ky, k2 = g.kx, g.ky, g.k2

        def place(v):
            o = np.where(bulk, v, 0.0)
            lv = np.where(line, v, 0.0)[:, 0]
            o[:, 0] += lv
            o[conj_rows, 0] += np.conj(lv)
            return o

        out: Dict[str, np.ndarray] = {}
        for a in range(n):
            out[f"Jpsi[{a}]_x"] = np.zeros((g.ny, g.hx), dtype=np.complex128)
            out[f"Jpsi[{a}]_y"] = np.zeros((g.ny, g.hx), dtype=np.complex128)
        for k in ("pi_xx", "pi_xy", "pi_yy"):
            out[k] = np.zeros((g.ny, g.hx), dtype=np.complex128)
        kbt = cfg.kBT * cfg.chi
        if cfg.noise_order_parameter and kbt != 0.0:
            pref = 2.0 * kbt * g.grid_size * g.grid_size / g.volume
            for a in range(n):
                M = cfg.mobility[a]
                if M == 0.0:
                    continue
                with np.errstate(divide="ignore", invalid="ignore"):
                    sig = np.sqrt(0.5 * pref * M * k2)
                    fx = np.where(bulk, 1j * (kx / k2) * sig * xi_psi[a], 0.0)
                    fy = np.where(use, 1j * (ky / k2) * sig * xi_psi[a], 0.0)
                out[f"Jpsi[{a}]_x"] = fx
                out[f"Jpsi[{a}]_y"] = place(fy)
        if cfg.noise_momentum and cfg.mode != "quiescent" and cfg.kBT != 0.0 and (cfg.eta != 0.0 or cfg.zeta != 0.0):
            s = math.sqrt(0.5 * 2.0 * cfg.kBT * g.grid_size * g.grid_size / g.volume)
            se, sz = math.sqrt(cfg.eta), math.sqrt(cfg.zeta)
            x1, x2, x3 = xi_j
            out["pi_xx"] = place(-s * (sz * x1 + se * x2))
            out["pi_yy"] = place(-s * (sz * x1 - se * x2))
            out["pi_xy"] = place(-s * se * x3)
        return out

    def step_with_flux_fields(self, u: np.ndarray, noise=None):
        """(next state, the step's flux buffer): stage fluxes weighted 1/6, 1/6, 2/3 (SRK3) or 1
        (Euler), the first draw's noise flux / sqrt(dt) ("philox" noise only), and in incompressible
        dynamics the projection pressure on pi_xx, pi_yy at k != 0 (time_integrator_*.h,
        buffer_flux.cc:170-226)."""
        cfg, g = self.cfg, self.geo
        step = self.step_index
        if cfg.integrator == "euler":
            stages, weights = [u], [1.0]
            out = self.step(u, noise)
        else:
            if noise == "philox":
                sa, sb = self.philox_noise(step)
            elif noise is None:
                sa = sb = np.zeros(self.shape, dtype=np.complex128)
            else:
                sa, sb = noise
            u1 = self._stage(u, u, sa + BETA[0] * sb, *STAGE_WEIGHTS[0])
            u2 = self._stage(u1, u, sa + BETA[1] * sb, *STAGE_WEIGHTS[1])
            out = self._stage(u2, u, sa + BETA[2] * sb, *STAGE_WEIGHTS[2])
            self.step_index += 1
            self.time += cfg.dt
            stages, weights = [u, u1, u2], [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]
        acc: Dict[str, np.ndarray] = {}
        for w, st in zip(weights, stages):
            for k, v in self.flux_fields(st).items():
                acc[k] = acc[k] + w * v if k in acc else w * v
        if noise == "philox":
            ids = self.mode_ids()
            xp = [philox_normals(cfg.noise_seed, self.member, step, psi_stream(a), ids)[0] for a in range(cfg.num_order_parameters)]
            xj = [philox_normals(cfg.noise_seed, self.member, step, j_stream(m), ids)[0] for m in range(3)]
            for k, v in self.noise_flux_fields(xp, xj).items():
                acc[k] = acc[k] + v / math.sqrt(cfg.dt)
        if cfg.mode == "incompressible":
            use = g.active & (g.k2 != 0.0)
            kx, ky, k2 = g.kx, g.ky, np.where(use, g.k2, 1.0)
            rx = -1j * (kx * acc["pi_xx"] + ky * acc["pi_xy"])
            ry = -1j * (kx * acc["pi_xy"] + ky * acc["pi_yy"])
            ph = np.where(use, -1j * (kx * rx + ky * ry) / k2, 0.0)
            acc["pi_xx"] = acc["pi_xx"] + ph
            acc["pi_yy"] = acc["pi_yy"] + ph
        return out, acc

    def noise_flux_xy(self, xi3: np.ndarray) -> np.ndarray:
        """pi_xy of one j_sto draw (fcalculator.cc:587-700): -s sqrt(eta) xi3 on the
        active k != 0 modes with gx > 0, and on the kx = 0 line the drawn half with
        its conjugate partner."""
        cfg, g = self.cfg, self.geo
        out = np.zeros((g.ny, g.hx), dtype=np.complex128)
        if not (cfg.noise_momentum and cfg.mode != "quiescent" and cfg.kBT != 0.0 and (cfg.eta != 0.0 or cfg.zeta != 0.0)):
            return out
        use = g.active & (g.k2 != 0.0)
        line = use & (g.gx == 0) & (g.gy < (g.ny - g.gy) % g.ny)
        bulk = use & (g.gx != 0)
        s = math.sqrt(0.5 * 2.0 * cfg.kBT * g.grid_size * g.grid_size / g.volume)
        pxy = -s * math.sqrt(cfg.eta) * xi3
        out = np.where(bulk, pxy, 0.0)
        lv = np.where(line, pxy, 0.0)[:, 0]
        conj_rows = (g.ny - np.arange(g.ny)) % g.ny
        out[:, 0] += lv
        out[conj_rows, 0] += np.conj(lv)
        return out

    def step_with_flux(self, u: np.ndarray, noise=None):
        """(next state, step flux pi_xy): the SRK3 stage-weighted deterministic flux
        (1/6, 1/6, 2/3; Euler 1) plus the first draw's stochastic flux / sqrt(dt)
        (time_integrator_srk3_compressible.h:99-146, buffer_flux.cc:170-195)."""
        cfg = self.cfg
        step = self.step_index
        flux = np.zeros((self.geo.ny, self.geo.hx), dtype=np.complex128)
        if cfg.integrator == "euler":
            flux += self.momentum_flux_xy(u)
            out = self.step(u, noise)
        else:
            noisy = cfg.noise_order_parameter or (cfg.noise_momentum and cfg.mode != "quiescent")
            if noise == "philox" and noisy:
                sa, sb = self.philox_noise(step)
            elif noise is None or not noisy:
                sa = sb = np.zeros(self.shape, dtype=np.complex128)
            else:
                sa, sb = noise
            u1 = self._stage(u, u, sa + BETA[0] * sb, *STAGE_WEIGHTS[0])
            u2 = self._stage(u1, u, sa + BETA[1] * sb, *STAGE_WEIGHTS[1])
            out = self._stage(u2, u, sa + BETA[2] * sb, *STAGE_WEIGHTS[2])
            for w, cur in zip((1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0), (u, u1, u2)):
                flux += w * self.momentum_flux_xy(cur)
            self.step_index += 1
            self.time += cfg.dt
        if noise == "philox":
            xa = philox_normals(cfg.noise_seed, self.member, step, j_stream(2), self.mode_ids())[0]
            flux += self.noise_flux_xy(xa) / math.sqrt(cfg.dt)
        return out, flux


def time_series_l2(cfg: Config, state: np.ndarray) -> Dict[str, float]:
    """Spectral L2 columns of TimeSeriesMeasure (measure_time_series.cc:233-275):
    cell_area / grid_size * sum over active modes but (0, 0) of w (k^2) |u|^2, w = 2 off kx = 0."""
    g = Geometry(cfg)
    use = g.active & ~((g.gx == 0) & (g.sgy == 0))
    w = np.where(g.gx == 0, 1.0, 2.0)
    pref = (g.volume / g.grid_size) / g.grid_size

    def s(f, k2=False):
        return float(pref * np.sum(np.where(use, w * (g.k2 if k2 else 1.0) * np.abs(f) ** 2, 0.0)))

    n = cfg.num_order_parameters
    out = {"|rho|^2": s(state[0]), "|d_rho|^2": s(state[0], True),
           "|j|^2": s(state[n + 1]) + s(state[n + 2]), "|d_j|^2": s(state[n + 1], True) + s(state[n + 2], True)}
    for a in range(n):
        out[f"|psi[{a}]|^2"] = s(state[1 + a])
        out[f"|d_psi[{a}]|^2"] = s(state[1 + a], True)
    return out


def time_series_energies(cfg: Config, state: np.ndarray) -> Dict[str, float]:
    """Energy columns of TimeSeriesMeasure (measure_time_series.cc:152-188, 305-470):

    E_K   compressible: sum over the padded grid of (jx^2 + jy^2) / (2 rho) dA (physical fields);
          incompressible: cell / (2 Ng rho0) sum over active modes of w (|jx|^2 + |jy|^2); quiescent: 0
    E_C   compressible with cT^2 != 0: cT^2 cell / (2 Ng rho0) sum over active modes but (0, 0) of w |rho|^2
    E_psi per order parameter cell / (2 Ng) sum over active modes of w (k0 + k2 k^2 + k4 k^4) |psi|^2,
          plus, for phi4 with some u != 0, sum over the padded grid of u psi^4 / 4 dA
    E_T   E_K + E_psi + E_C
    with w = 2 off the kx = 0 line, rho0 = Re rho(0) / Ng, dA = cell = V / Ng.
    """
    g = Geometry(cfg)
    n = cfg.num_order_parameters
    w = np.where(g.gx == 0, 1.0, 2.0)
    act = g.active
    cell = g.volume / g.grid_size
    rho0 = state[0, 0, 0].real / g.grid_size
    mode = cfg.mode
    kin = 0.0
    if mode == "compressible":
        rho, jx, jy = g.backward(state[0]), g.backward(state[n + 1]), g.backward(state[n + 2])
        kin = float(np.sum(0.5 * (jx * jx + jy * jy) / rho * cell))
    elif mode == "incompressible":
        kin = 0.5 * cell / (g.grid_size * rho0) * float(np.sum(np.where(act, w * (np.abs(state[n + 1]) ** 2 + np.abs(state[n + 2]) ** 2), 0.0)))
    comp = 0.0
    if mode == "compressible" and cfg.cT * cfg.cT != 0.0:
        use = act & ~((g.gx == 0) & (g.sgy == 0))
        comp = 0.5 * cfg.cT * cfg.cT * cell / (g.grid_size * rho0) * float(np.sum(np.where(use, w * np.abs(state[0]) ** 2, 0.0)))
    free = 0.0
    for a in range(n):
        if cfg.free_energy == "phi4" or cfg.free_energy in PLUGINS:
            k0, k2c, k4 = cfg.phi4_a[a], cfg.phi4_b[a], 0.0
        elif cfg.free_energy == "quadratic":
            k0, k2c, k4 = cfg.quad_a[a], 0.0, 0.0
        else:
            k0 = k2c = k4 = 0.0
        if k0 == 0.0 and k2c == 0.0 and k4 == 0.0:
            continue
        coef = k0 + k2c * g.k2 + k4 * g.k2 * g.k2
        free += 0.5 * cell / g.grid_size * float(np.sum(np.where(act, w * coef * np.abs(state[1 + a]) ** 2, 0.0)))
    if cfg.free_energy in PLUGINS and n > 0:
        free += float(np.sum(cfg.physical_density([g.backward(state[1 + a]) for a in range(n)]) * cell))
    elif cfg.free_energy == "phi4" and any(u != 0.0 for u in cfg.phi4_u):
        dens = np.zeros((g.ny, g.nx))
        for a in range(n):
            p = g.backward(state[1 + a])
            dens += 0.25 * cfg.phi4_u[a] * p ** 4
        free += float(np.sum(dens * cell))
    return {"E_T": kin + free + comp, "E_K": kin, "E_psi": free, "E_C": comp}


def green_kubo_modes(cfg: Config, selection: str = "diagonal") -> List[Tuple[int, int]]:
    """Wave numbers (nx, ny) of measure_yokota_green_kubo.cc:42-96."""
    max_nx = max(0, cfg.active[0] // 2 - 1)
    max_ny = max(0, cfg.active[1] // 2 - 1)
    if selection == "diagonal":
        return [(n, n) for n in range(1, min(max_nx, max_ny) + 1)]
    out = [(0, n) for n in range(1, max_ny + 1)]
    for nx in range(1, max_nx + 1):
        for ny in range(-max_ny, max_ny + 1):
            out.append((nx, ny))
    return out


class GreenKubo:
    """YokotaGreenKuboMeasure::observe (measure_yokota_green_kubo.cc:128-190) over
    a step flux pi_xy given per step; S sums per (tau, mode) and completed blocks."""

    def __init__(self, cfg: Config, nevery: int, nblock: int, selection: str = "diagonal", kBT: Optional[float] = None):
        self.cfg = cfg
        self.geo = Geometry(cfg)
        self.nevery, self.nblock = nevery, nblock
        self.ntau = nblock // nevery
        self.kBT = cfg.kBT if kBT is None else kBT
        self.modes = green_kubo_modes(cfg, selection)
        g = self.geo
        self.index = [(ny % g.ny, nx) for nx, ny in self.modes]
        self.integrals = np.zeros(len(self.modes), dtype=np.complex128)
        self.sums = np.zeros((self.ntau, len(self.modes)))
        self.block_step = 0
        self.nsample = 0

    def observe(self, flux: np.ndarray) -> None:
        self.block_step += 1
        area = self.geo.volume
        cell_area = area / self.geo.grid_size
        wdt = 0.5 * self.cfg.dt if self.block_step == 1 else self.cfg.dt
        self.integrals += wdt * cell_area * np.array([flux[gy, gx] for gy, gx in self.index])
        if self.block_step % self.nevery == 0:
            ti = self.block_step // self.nevery - 1
            tau = self.block_step * self.cfg.dt
            self.sums[ti] += np.abs(self.integrals) ** 2 / (2.0 * tau * self.kBT * area)
        if self.block_step == self.nblock:
            self.nsample += 1
            self.block_step = 0
            self.integrals[:] = 0.0


# --------------------------------------------------------------------------
# layout helpers shared by the tests
# --------------------------------------------------------------------------
def ref_to_active(cfg: Config, u: np.ndarray) -> np.ndarray:
    """Reference State layout -> active layout [field, gx, j] (j: ky = 0..Nay/2-1, then -(Nay/2-1)..-1)."""
    g = Geometry(cfg)
    rows = active_rows(cfg)
    return np.ascontiguousarray(u[:, rows, : g.nax // 2].transpose(0, 2, 1))


def active_rows(cfg: Config) -> np.ndarray:
    nx, ny = cfg.grid
    nay = cfg.active[1]
    pos = np.arange(nay // 2)
    neg = np.arange(-(nay // 2 - 1), 0)
    return np.concatenate([pos, ny + neg])


def active_to_ref(cfg: Config, a: np.ndarray) -> np.ndarray:
    g = Geometry(cfg)
    out = np.zeros((a.shape[0], g.ny, g.hx), dtype=np.complex128)
    out[:, active_rows(cfg), : g.nax // 2] = a.transpose(0, 2, 1)
    return out


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    den = np.linalg.norm(b.ravel())
    num = np.linalg.norm((a - b).ravel())
    return float(num / den) if den > 0 else float(num)
