"""Python binding of the B200 step engine (ctypes over lib/libshhd_b200.so).

The engine is the CUDA path; this module only moves arguments across the C
ABI declared in include/shhd_b200.h.  Importing it loads the library and
fails loudly if it has not been built (there is no CPU fallback).

Typical use mirrors the reference's driver loop (src/project.h:128-145)::

    cfg = config_from_script(open("input.script").read())
    eng = Engine(cfg)
    eng.set_state(state)          # reference State layout, complex128
    eng.step(100)                 # FluidSolver::step x 100
    state = eng.get_state()
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libshhd_b200.so")

MAX_OP = 8
MAX_FORCES = 8
MAX_FE_PARAMS = 4

SHHD_OK = 0
SHHD_EINVAL = -1
SHHD_ECUDA = -2
SHHD_ENOMEM = -3
SHHD_ENUMERIC = -4
SHHD_EUNSUPPORTED = -5

COMPRESSIBLE, INCOMPRESSIBLE, QUIESCENT = 0, 1, 2
EULER, SRK3 = 0, 1
FP64, FP32 = 0, 1
NOISE_PHILOX, NOISE_EXTERNAL = 0, 1


class SineForce(ctypes.Structure):
    _fields_ = [("target", ctypes.c_int), ("component", ctypes.c_int), ("axis", ctypes.c_int), ("nk", ctypes.c_int),
                ("amplitude", ctypes.c_double)]


class GradientForce(ctypes.Structure):
    _fields_ = [("component", ctypes.c_int), ("direction", ctypes.c_int), ("amplitude", ctypes.c_double)]


class Config(ctypes.Structure):
    """Mirror of shhd_config."""
    _fields_ = [
        ("active_nx", ctypes.c_int), ("active_ny", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("lx", ctypes.c_double), ("ly", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("mode", ctypes.c_int), ("integrator", ctypes.c_int),
        ("num_order_parameters", ctypes.c_int),
        ("free_energy", ctypes.c_int),
        ("mu_k0", ctypes.c_double * MAX_OP), ("mu_k2", ctypes.c_double * MAX_OP),
        ("mu_k4", ctypes.c_double * MAX_OP), ("mu_u3", ctypes.c_double * MAX_OP),
        ("cT", ctypes.c_double),
        ("eta", ctypes.c_double), ("zeta", ctypes.c_double),
        ("mobility", ctypes.c_double * MAX_OP),
        ("momentum_advection", ctypes.c_int), ("order_parameter_advection", ctypes.c_int),
        ("noise_momentum", ctypes.c_int), ("noise_order_parameter", ctypes.c_int),
        ("noise_seed", ctypes.c_int64),
        ("kBT", ctypes.c_double), ("chi", ctypes.c_double),
        ("n_sine_forces", ctypes.c_int), ("sine_forces", SineForce * MAX_FORCES),
        ("n_gradient_forces", ctypes.c_int), ("gradient_forces", GradientForce * MAX_FORCES),
        ("precision", ctypes.c_int), ("noise_source", ctypes.c_int),
        ("batch", ctypes.c_int), ("member_offset", ctypes.c_int),
        ("fe_plugin", ctypes.c_int), ("fe_param", (ctypes.c_double * MAX_OP) * MAX_FE_PARAMS),
    ]

    def copy(self) -> "Config":
        c = Config()
        ctypes.memmove(ctypes.byref(c), ctypes.byref(self), ctypes.sizeof(Config))
        return c


class Info(ctypes.Structure):
    _fields_ = [
        ("nfields", ctypes.c_int), ("state_doubles", ctypes.c_size_t), ("active_modes", ctypes.c_size_t),
        ("n_inverse", ctypes.c_int), ("n_forward", ctypes.c_int), ("n_evolved", ctypes.c_int),
        ("device_bytes", ctypes.c_size_t), ("bytes_per_stage", ctypes.c_double), ("fft_flops_per_stage", ctypes.c_double),
        ("step_index", ctypes.c_int64), ("time", ctypes.c_double),
    ]


class InitialField(ctypes.Structure):
    """Mirror of shhd_initial_field (one device-generated initial field)."""
    _fields_ = [
        ("style", ctypes.c_int), ("channel", ctypes.c_int), ("seed", ctypes.c_uint64),
        ("mean", ctypes.c_double), ("s0", ctypes.c_double), ("c0", ctypes.c_double), ("c2", ctypes.c_double),
        ("c4", ctypes.c_double), ("amplitude", ctypes.c_double), ("rho0", ctypes.c_double),
        ("n0", ctypes.c_double), ("sigma", ctypes.c_double), ("x0", ctypes.c_double), ("y0", ctypes.c_double),
        ("sigma_x", ctypes.c_double), ("sigma_y", ctypes.c_double), ("nkx", ctypes.c_int), ("nky", ctypes.c_int),
    ]

    @classmethod
    def of(cls, spec) -> "InitialField":
        if isinstance(spec, cls):
            return spec
        f = cls()
        for name, _t in cls._fields_:
            v = spec[name]
            setattr(f, name, int(v) & 0xFFFFFFFFFFFFFFFF if name == "seed" else v)
        return f


class ShhdError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


# every symbol include/shhd_b200.h declares
EXPORTED = (
    "shhd_last_error", "shhd_config_default", "shhd_config_from_script", "shhd_engine_create", "shhd_engine_destroy",
    "shhd_engine_info", "shhd_engine_set_state", "shhd_engine_get_state", "shhd_engine_step", "shhd_engine_step_async",
    "shhd_engine_synchronize", "shhd_engine_set_external_noise", "shhd_engine_rhs", "shhd_engine_set_time",
    "shhd_engine_stream", "shhd_engine_state_device", "shhd_engine_set_profiling", "shhd_engine_kernel_stats",
    "shhd_engine_reset_stats", "shhd_engine_set_member", "shhd_rhs_noalloc", "shhd_engine_set_graph_chunk",
    "shhd_engine_sk_accumulate", "shhd_engine_sk_read", "shhd_engine_autotune",
    "shhd_engine_gk_enable", "shhd_engine_gk_read", "shhd_engine_l2_sums", "shhd_engine_set_gaussian_field",
    "shhd_engine_set_initial_field", "shhd_engine_check_transverse", "shhd_engine_energies",
    "shhd_engine_flux0_enable", "shhd_engine_flux0_read", "shhd_engine_profile_line", "shhd_engine_profile_velocity",
    "shhd_engine_flux_line_enable", "shhd_engine_flux_line_read", "shhd_engine_flux_tap_schedule",
    "shhd_engine_set_family", "shhd_engine_family", "shhd_engine_set_launch_shape", "shhd_engine_launch_shape",
    "shhd_free_energy_plugin_count", "shhd_free_energy_plugin_name", "shhd_free_energy_plugin_key",
)

FAMILY_NAMES = {0: "single-line", 1: "pair-line", 2: "pair-line + register row pass", 3: "pair-line + split row pass",
                4: "pair-line + two-pair row pass"}

KERNEL_KINDS = ("col_inverse", "row_pass", "col_forward", "other")


def _load() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is not built; run `make -C {os.path.dirname(LIB_PATH)}/..` (the engine has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    vp, dp, sz, i = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_size_t, ctypes.c_int
    lib.shhd_last_error.restype = ctypes.c_char_p
    lib.shhd_config_default.argtypes = [ctypes.POINTER(Config)]
    lib.shhd_config_from_script.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config)]
    lib.shhd_engine_create.argtypes = [ctypes.POINTER(Config), ctypes.POINTER(vp)]
    lib.shhd_engine_destroy.argtypes = [vp]
    lib.shhd_engine_destroy.restype = None
    lib.shhd_engine_info.argtypes = [vp, ctypes.POINTER(Info)]
    lib.shhd_engine_set_state.argtypes = [vp, i, dp, sz]
    lib.shhd_engine_get_state.argtypes = [vp, i, dp, sz]
    lib.shhd_engine_step.argtypes = [vp, i]
    lib.shhd_engine_step_async.argtypes = [vp, i]
    lib.shhd_engine_synchronize.argtypes = [vp]
    lib.shhd_engine_set_external_noise.argtypes = [vp, i, dp, dp, sz]
    lib.shhd_engine_rhs.argtypes = [vp, i, dp, sz]
    lib.shhd_engine_set_time.argtypes = [vp, ctypes.c_int64, ctypes.c_double]
    lib.shhd_engine_stream.argtypes = [vp]
    lib.shhd_engine_stream.restype = vp
    lib.shhd_engine_state_device.argtypes = [vp]
    lib.shhd_engine_state_device.restype = vp
    lib.shhd_engine_set_profiling.argtypes = [vp, i]
    lib.shhd_engine_kernel_stats.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_double)]
    lib.shhd_engine_reset_stats.argtypes = [vp]
    lib.shhd_engine_set_member.argtypes = [vp, i, ctypes.c_uint32, ctypes.c_int64, ctypes.c_double, i]
    lib.shhd_rhs_noalloc.argtypes = [ctypes.POINTER(Config), vp, vp, sz, vp]
    lib.shhd_engine_set_graph_chunk.argtypes = [vp, i]
    lib.shhd_engine_sk_accumulate.argtypes = [vp, i]
    lib.shhd_engine_sk_read.argtypes = [vp, dp, sz, ctypes.POINTER(ctypes.c_int64), i]
    lib.shhd_engine_autotune.argtypes = [vp, i, ctypes.POINTER(i), ctypes.POINTER(i), dp]
    lib.shhd_engine_set_family.argtypes = [vp, i]
    lib.shhd_engine_family.argtypes = [vp]
    lib.shhd_engine_set_launch_shape.argtypes = [vp, i, i]
    lib.shhd_engine_launch_shape.argtypes = [vp, ctypes.POINTER(i), ctypes.POINTER(i)]
    lib.shhd_free_energy_plugin_count.argtypes = []
    lib.shhd_free_energy_plugin_name.argtypes = [i]
    lib.shhd_free_energy_plugin_name.restype = ctypes.c_char_p
    lib.shhd_free_energy_plugin_key.argtypes = [i, i]
    lib.shhd_free_energy_plugin_key.restype = ctypes.c_char_p
    lib.shhd_engine_gk_enable.argtypes = [vp, i, i, i]
    lib.shhd_engine_gk_read.argtypes = [vp, i, dp, sz, ctypes.POINTER(ctypes.c_int64), i]
    lib.shhd_engine_l2_sums.argtypes = [vp, i, dp, sz]
    d = ctypes.c_double
    lib.shhd_engine_set_gaussian_field.argtypes = [vp, i, i, ctypes.c_uint64, i, d, d, d, d, d]
    lib.shhd_engine_set_initial_field.argtypes = [vp, i, i, ctypes.POINTER(InitialField)]
    lib.shhd_engine_check_transverse.argtypes = [vp, ctypes.POINTER(InitialField), ctypes.POINTER(InitialField)]
    lib.shhd_engine_energies.argtypes = [vp, i, dp, sz]
    lib.shhd_engine_flux0_enable.argtypes = [vp]
    lib.shhd_engine_flux0_read.argtypes = [vp, i, dp, sz]
    lib.shhd_engine_profile_line.argtypes = [vp, i, i, i, dp, sz]
    lib.shhd_engine_profile_velocity.argtypes = [vp, i, i, i, dp, sz]
    lib.shhd_engine_flux_line_enable.argtypes = [vp, i]
    lib.shhd_engine_flux_line_read.argtypes = [vp, i, i, dp, sz]
    lib.shhd_engine_flux_tap_schedule.argtypes = [vp, i, ctypes.c_int64, ctypes.c_int64]
    return lib


lib = _load()


def _check(rc: int) -> None:
    if rc != SHHD_OK:
        raise ShhdError(rc, lib.shhd_last_error().decode())


def default_config() -> Config:
    c = Config()
    _check(lib.shhd_config_default(ctypes.byref(c)))
    return c


def free_energy_plugins() -> dict:
    """The free-energy plugin styles compiled into the library: {name: (id, [parameter keys])}."""
    out = {}
    for sid in range(1, lib.shhd_free_energy_plugin_count() + 1):
        keys, k = [], 0
        while (key := lib.shhd_free_energy_plugin_key(sid, k)) is not None:
            keys.append(key.decode())
            k += 1
        out[lib.shhd_free_energy_plugin_name(sid).decode()] = (sid, keys)
    return out


def config_from_script(text: str) -> Config:
    """Parse a reference input script into a Config (host only)."""
    c = Config()
    _check(lib.shhd_config_from_script(text.encode(), ctypes.byref(c)))
    return c


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Engine:
    """One engine: `cfg.batch` members of one configuration on the current GPU."""

    def __init__(self, cfg: Config):
        self.cfg = cfg.copy()
        h = ctypes.c_void_p()
        _check(lib.shhd_engine_create(ctypes.byref(self.cfg), ctypes.byref(h)))
        self._h = h
        self.info = self.get_info()
        self.shape = (self.info.nfields, cfg.ny, cfg.nx // 2 + 1)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            lib.shhd_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def get_info(self) -> Info:
        inf = Info()
        _check(lib.shhd_engine_info(self._h, ctypes.byref(inf)))
        return inf

    def _as_ref(self, state: np.ndarray) -> np.ndarray:
        a = np.ascontiguousarray(state, dtype=np.complex128)
        if a.shape != self.shape:
            raise ValueError(f"state shape {a.shape} != {self.shape}")
        return a

    def set_state(self, state: np.ndarray, member: int = 0) -> None:
        a = self._as_ref(state)
        _check(lib.shhd_engine_set_state(self._h, member, _dptr(a.view(np.float64)), a.size * 2))

    def get_state(self, member: int = 0, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.shape, dtype=np.complex128)
        elif out.shape != self.shape or out.dtype != np.complex128 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous complex128 array of the state shape")
        _check(lib.shhd_engine_get_state(self._h, member, _dptr(out.view(np.float64)), out.size * 2))
        return out

    def step(self, nsteps: int = 1) -> None:
        _check(lib.shhd_engine_step(self._h, nsteps))

    def step_async(self, nsteps: int = 1) -> None:
        _check(lib.shhd_engine_step_async(self._h, nsteps))

    def synchronize(self) -> None:
        _check(lib.shhd_engine_synchronize(self._h))

    def set_external_noise(self, sto_a: np.ndarray, sto_b: Optional[np.ndarray] = None, member: int = 0) -> None:
        a = self._as_ref(sto_a)
        b = self._as_ref(sto_b) if sto_b is not None else None
        _check(lib.shhd_engine_set_external_noise(self._h, member, _dptr(a.view(np.float64)),
                                                  _dptr(b.view(np.float64)) if b is not None else None, a.size * 2))

    def rhs(self, member: int = 0) -> np.ndarray:
        out = np.zeros(self.shape, dtype=np.complex128)
        _check(lib.shhd_engine_rhs(self._h, member, _dptr(out.view(np.float64)), out.size * 2))
        return out

    def set_time(self, step_index: int, time: float) -> None:
        _check(lib.shhd_engine_set_time(self._h, int(step_index), float(time)))

    def set_member(self, member: int, key: int, step_origin: int = 0, noise_scale: float = 1.0, active: bool = True) -> None:
        """Per-member noise key, step origin, amplitude factor and active flag (serving)."""
        _check(lib.shhd_engine_set_member(self._h, member, int(key) & 0xFFFFFFFF, int(step_origin), float(noise_scale), 1 if active else 0))

    def set_graph_chunk(self, chunk: int) -> None:
        """Replay captured CUDA graphs of `chunk` steps (0: direct launches)."""
        _check(lib.shhd_engine_set_graph_chunk(self._h, int(chunk)))

    def sk_accumulate(self, field: int) -> None:
        """Add one FP64 sample of S(k) = V <|u_k|^2> / Np^4 (mean over active members) on the device."""
        _check(lib.shhd_engine_sk_accumulate(self._h, int(field)))

    def sk_read(self, reset: bool = True):
        """(sum of the S(k) samples as [gx, j] in the engine's mode order, number of samples)."""
        n = self.info.active_modes
        out = np.zeros(n, dtype=np.float64)
        cnt = ctypes.c_int64()
        _check(lib.shhd_engine_sk_read(self._h, _dptr(out), n, ctypes.byref(cnt), 1 if reset else 0))
        return out.reshape(self.cfg.active_nx // 2, self.cfg.active_ny - 1), int(cnt.value)

    def autotune(self, trial_steps: int = 3) -> dict:
        """Time the valid kernel families x {direct, graph} on the current state, then the launch
        shapes of the chosen family's pair-line kernels; keep the fastest."""
        fam, chunk = ctypes.c_int(), ctypes.c_int()
        ms = np.full(10, np.nan)
        _check(lib.shhd_engine_autotune(self._h, int(trial_steps), ctypes.byref(fam), ctypes.byref(chunk), _dptr(ms)))
        row, col = self.launch_shape
        return {"family": FAMILY_NAMES[fam.value], "graph_chunk": chunk.value,
                "ms_per_step": [None if np.isnan(x) else float(x) for x in ms],
                "launch_shape": {"row_blocks": row, "col_blocks": col}}

    def set_family(self, family: int) -> None:
        """Kernel family: -1 default, 0 single-line, 1 pair-line, 2 pair-line with the register row pass,
        3 pair-line with the split row pass, 4 pair-line with the two-pair row pass."""
        _check(lib.shhd_engine_set_family(self._h, int(family)))

    @property
    def family(self) -> int:
        return int(lib.shhd_engine_family(self._h))

    def set_launch_shape(self, row_blocks: int = 0, col_blocks: int = 0) -> None:
        """Blocks per SM the pair-line row pass (2 or 3) and column forward (3 or 4) are compiled
        for; 0 keeps the rule."""
        _check(lib.shhd_engine_set_launch_shape(self._h, int(row_blocks), int(col_blocks)))

    @property
    def launch_shape(self) -> Tuple[int, int]:
        """(row-pass, column-forward) blocks per SM in use; 0 where the kernel is not a pair-line one."""
        r, c = ctypes.c_int(), ctypes.c_int()
        _check(lib.shhd_engine_launch_shape(self._h, ctypes.byref(r), ctypes.byref(c)))
        return r.value, c.value

    def set_gaussian_field(self, member: int, field: int, seed: int, channel: int, mean: float, s0: float,
                           c0: float = 1.0, c2: float = 0.0, c4: float = 0.0) -> None:
        """Write one field on the device: sigma(k) xi_k per active mode, `mean` at k = 0."""
        _check(lib.shhd_engine_set_gaussian_field(self._h, int(member), int(field), int(seed) & 0xFFFFFFFFFFFFFFFF, int(channel),
                                                  float(mean), float(s0), float(c0), float(c2), float(c4)))

    def set_initial_field(self, member: int, field: int, spec) -> None:
        """Generate one field on the device from an InitialField (or a dict of its fields)."""
        f = InitialField.of(spec)
        _check(lib.shhd_engine_set_initial_field(self._h, int(member), int(field), ctypes.byref(f)))

    def check_transverse(self, jx, jy) -> None:
        """Raise ShhdError unless the two momentum specs are transverse at every active k != 0 (FP64)."""
        a, b = InitialField.of(jx), InitialField.of(jy)
        _check(lib.shhd_engine_check_transverse(self._h, ctypes.byref(a), ctypes.byref(b)))

    def time_series_energies(self, member: int = 0) -> dict:
        """The reference time-series measure's energy columns of the current state (FP64 sums)."""
        raw = np.zeros(4, dtype=np.float64)
        _check(lib.shhd_engine_energies(self._h, int(member), _dptr(raw), raw.size))
        return {"E_T": float(raw[0]), "E_K": float(raw[1]), "E_psi": float(raw[2]), "E_C": float(raw[3])}

    def flux0_enable(self, every: int = 1, phase: int = 0) -> None:
        """Record the k = 0 flux columns from now on, on the steps s = phase mod every (see flux_tap_request)."""
        _check(lib.shhd_engine_flux0_enable(self._h))
        self.flux_tap_request(0, every, phase)

    def flux_tap_request(self, tap: int, every: int, phase: int) -> None:
        """Ask tap 0 (k = 0), 1 (ky = 0 line) or 2 (kx = 0 line) to record the steps s = phase mod every
        (s: the engine step index after the step).  Requests accumulate: the tap records every step any
        request needs (period gcd(every, every', phase - phase'))."""
        import math
        sched = self.__dict__.setdefault("_tap_schedules", {})
        ph = phase % every
        if tap in sched:
            p0, q0 = sched[tap]
            g = math.gcd(math.gcd(p0, every), abs(ph - q0))
            self.flux_tap_schedule(tap, g, q0)
        else:
            self.flux_tap_schedule(tap, every, ph)

    def flux_tap_schedule(self, tap: int, every: int, phase: int) -> None:
        """Set the steps a tap records (s = phase mod every), replacing earlier requests."""
        self.__dict__.setdefault("_tap_schedules", {})[tap] = (int(every), int(phase) % int(every))
        _check(lib.shhd_engine_flux_tap_schedule(self._h, int(tap), int(every), int(phase)))

    def flux0_read(self, member: int = 0) -> dict:
        """The last step's k = 0 flux columns: pi_xx, pi_xy, pi_yy, Jpsi[a]_x, Jpsi[a]_y."""
        n = self.cfg.num_order_parameters
        raw = np.zeros(3 + 2 * n, dtype=np.float64)
        _check(lib.shhd_engine_flux0_read(self._h, int(member), _dptr(raw), raw.size))
        out = {"pi_xx": raw[0], "pi_xy": raw[1], "pi_yy": raw[2]}
        for a in range(n):
            out[f"Jpsi[{a}]_x"] = raw[3 + 2 * a]
            out[f"Jpsi[{a}]_y"] = raw[4 + 2 * a]
        return {k: float(v) for k, v in out.items()}

    def profile_line(self, field: int, axis: int, member: int = 0) -> np.ndarray:
        """The spectral line of `field` an ave/profile along `axis` needs (complex128): axis 0 the
        ky = 0 row over the active kx, axis 1 the kx = 0 column in the engine's ky order."""
        n = self.cfg.active_nx // 2 if axis == 0 else self.cfg.active_ny - 1
        raw = np.zeros(2 * n, dtype=np.float64)
        _check(lib.shhd_engine_profile_line(self._h, int(member), int(field), int(axis), _dptr(raw), raw.size))
        return raw.view(np.complex128)

    def profile_velocity(self, component: int, axis: int, member: int = 0) -> np.ndarray:
        """The compressible velocity component j_c / rho summed over the transverse axis (FP64)."""
        n = self.cfg.nx if axis == 0 else self.cfg.ny
        raw = np.zeros(n, dtype=np.float64)
        _check(lib.shhd_engine_profile_velocity(self._h, int(member), int(component), int(axis), _dptr(raw), raw.size))
        return raw

    def flux_line_enable(self, axis: int, every: int = 1, phase: int = 0) -> None:
        """Record the step's flux buffer along the ky = 0 row (axis 0) or kx = 0 column (axis 1), on the
        steps s = phase mod every (see flux_tap_request)."""
        _check(lib.shhd_engine_flux_line_enable(self._h, int(axis)))
        self.flux_tap_request(1 + int(axis), every, phase)

    def flux_line(self, axis: int, member: int = 0) -> dict:
        """The last step's fluxes along the line, {pi_xx, pi_xy, pi_yy, Jpsi[a]_x, Jpsi[a]_y: complex128}."""
        n = self.cfg.num_order_parameters
        nline = self.cfg.active_nx // 2 if axis == 0 else self.cfg.active_ny - 1
        raw = np.zeros(2 * (3 + 2 * n) * nline, dtype=np.float64)
        _check(lib.shhd_engine_flux_line_read(self._h, int(axis), int(member), _dptr(raw), raw.size))
        z = raw.view(np.complex128).reshape(3 + 2 * n, nline)
        names = ["pi_xx", "pi_xy", "pi_yy"] + [f"Jpsi[{a}]_{d}" for a in range(n) for d in "xy"]
        return {k: z[c].copy() for c, k in enumerate(names)}

    def time_series_l2(self, member: int = 0) -> dict:
        """The reference time-series measure's spectral L2 columns of the current state (FP64)."""
        nf = self.info.nfields
        raw = np.zeros(2 * nf, dtype=np.float64)
        _check(lib.shhd_engine_l2_sums(self._h, int(member), _dptr(raw), raw.size))
        n = nf - 3
        out = {"|rho|^2": raw[0], "|d_rho|^2": raw[1], "|j|^2": raw[2 * (n + 1)] + raw[2 * (n + 2)],
               "|d_j|^2": raw[2 * (n + 1) + 1] + raw[2 * (n + 2) + 1]}
        for a in range(n):
            out[f"|psi[{a}]|^2"] = raw[2 * (1 + a)]
            out[f"|d_psi[{a}]|^2"] = raw[2 * (1 + a) + 1]
        return {k: float(v) for k, v in out.items()}

    def gk_enable(self, nevery: int, nblock: int, selection: str = "diagonal") -> None:
        """Start the Yokota-Green-Kubo stress measure (FP64, on the device)."""
        sel = {"diagonal": 0, "all": 1}[selection]
        _check(lib.shhd_engine_gk_enable(self._h, int(nevery), int(nblock), sel))
        mx, my = max(0, self.cfg.active_nx // 2 - 1), max(0, self.cfg.active_ny // 2 - 1)
        if sel == 0:
            self.gk_modes = [(n, n) for n in range(1, min(mx, my) + 1)]
        else:
            self.gk_modes = [(0, n) for n in range(1, my + 1)] + [(nx, ny) for nx in range(1, mx + 1) for ny in range(-my, my + 1)]
        self.gk_ntau = nblock // nevery

    def gk_read(self, member: int = 0, reset: bool = False):
        """(sums [tau, mode] of |I|^2 / (2 tau kBT V), completed blocks); S_mean = sums / blocks."""
        out = np.zeros((self.gk_ntau, len(self.gk_modes)), dtype=np.float64)
        cnt = ctypes.c_int64()
        _check(lib.shhd_engine_gk_read(self._h, int(member), _dptr(out), out.size, ctypes.byref(cnt), 1 if reset else 0))
        return out, int(cnt.value)

    def set_profiling(self, on: bool) -> None:
        _check(lib.shhd_engine_set_profiling(self._h, 1 if on else 0))

    def kernel_stats(self) -> dict:
        """{kind: (total_ms, launches, algorithmic_bytes)} since the last reset."""
        ms = (ctypes.c_double * 4)()
        n = (ctypes.c_int64 * 4)()
        by = (ctypes.c_double * 4)()
        _check(lib.shhd_engine_kernel_stats(self._h, ms, n, by))
        return {KERNEL_KINDS[k]: (ms[k], n[k], by[k]) for k in range(4)}

    def reset_stats(self) -> None:
        _check(lib.shhd_engine_reset_stats(self._h))

    @property
    def stream(self) -> int:
        return lib.shhd_engine_stream(self._h) or 0

    @property
    def state_device_ptr(self) -> int:
        return lib.shhd_engine_state_device(self._h) or 0
