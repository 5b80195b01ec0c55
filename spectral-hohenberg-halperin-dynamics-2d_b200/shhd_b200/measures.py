"""The reference's `measure` commands over an engine, written in the reference's file formats.

  time_series (measure_time_series.cc:109-286): the energy columns E_T E_K E_psi E_C
      (shhd_engine_energies) and the spectral L2 columns |rho|^2 ... |d_psi[a]|^2
      (shhd_engine_l2_sums), FP64 sums on the device; one line per observed step,
      `step time v...` in scientific notation with 16 digits.  The k = 0 flux
      columns pi_xx pi_xy pi_yy Jpsi[a]_x Jpsi[a]_y come from the engine's flux
      tap (shhd_engine_flux0_*), enabled when a column asks for it: the last
      step's stage-weighted (0, 0) fluxes, as the reference's flux buffer holds.
  ave/profile (measure_ave_profile.cc:180-453): block or running averages of
      field and flux profiles over one axis (class AveProfile).
  yokota_green_kubo (measure_yokota_green_kubo.cc:16-225): the stress
      autocorrelation table, accumulated on the device (class YokotaGreenKubo).
  snapshot (measure_snapshot.cc:43-138): `<file>_step<step>.snapshot`, the step
      zero-padded to the digits of the script's total run steps; space physical
      (every field inverse-transformed on the padded grid, rows gy-major) or
      spectral (the full R2C array, real and imaginary parts).

`run_script_measures` drives an engine through a script's `run` commands and
observes after every step, as Project::run_steps does (project.h:127-143).
"""
from __future__ import annotations

import re
from typing import Dict, List, Optional, TextIO

import numpy as np

_ENERGY = ("E_T", "E_K", "E_psi", "E_C")
_L2 = ("|rho|^2", "|d_rho|^2", "|j|^2", "|d_j|^2")
_PI = ("pi_xx", "pi_xy", "pi_yy")
_JPSI = re.compile(r"^Jpsi\[(\d+)\]_[xy]$")
_PSI_L2 = re.compile(r"^\|(d_)?psi\[(\d+)\]\|\^2$")


def _sci(v: float) -> str:
    return f"{v:.16e}"


class TimeSeries:
    """`measure <id> time_series on nevery N file F target ...` over one engine member."""

    def __init__(self, engine, file: str, nevery: int, targets: List[str], member: int = 0):
        if nevery <= 0:
            raise ValueError("time_series measure: nevery must be positive.")
        nop = engine.cfg.num_order_parameters
        for t in targets:
            m = _PSI_L2.match(t)
            j = _JPSI.match(t)
            a = int(m.group(2)) if m else (int(j.group(1)) if j else None)
            if a is not None and not 0 <= a < nop:
                raise ValueError(f"time_series target order-parameter index out of range: {t}")
            if not (t in _ENERGY or t in _L2 or t in _PI or a is not None):
                raise ValueError(f"unknown time_series target: {t}")
        self._flux = any(t in _PI or _JPSI.match(t) for t in targets)
        if self._flux:
            engine.flux0_enable(every=int(nevery), phase=0)   # observed at step % nevery == 0
        self.engine, self.file, self.nevery, self.targets, self.member = engine, file, int(nevery), list(targets), member
        self._out: Optional[TextIO] = None

    def _open(self) -> TextIO:
        if self._out is None:
            self._out = open(self.file, "w")
            self._out.write("# measure time_series\n")
            self._out.write("# step time" + "".join(" " + t for t in self.targets) + "\n")
        return self._out

    def values(self) -> Dict[str, float]:
        """The requested columns of the engine member's current state."""
        vals: Dict[str, float] = {}
        if any(t in _ENERGY for t in self.targets):
            vals.update(self.engine.time_series_energies(self.member))
        if any(t in _L2 or _PSI_L2.match(t) for t in self.targets):
            vals.update(self.engine.time_series_l2(self.member))
        if self._flux:
            vals.update(self.engine.flux0_read(self.member))
        return {t: vals[t] for t in self.targets}

    def observe(self, step: int, time: float) -> None:
        if step % self.nevery != 0:
            return
        out = self._open()
        v = self.values()
        out.write(f"{step} {_sci(time)}" + "".join(" " + _sci(v[t]) for t in self.targets) + "\n")
        out.flush()

    def close(self) -> None:
        if self._out is not None:
            self._out.close()
            self._out = None


def snapshot_filename(prefix: str, step: int, total_steps: int) -> str:
    """measure_snapshot.cc:34-52: one digit more than the total run steps have."""
    digits, n = 1, total_steps
    while n >= 10:
        n //= 10
        digits += 1
    return f"{prefix}_step{step:0{digits + 1}d}.snapshot"


def write_snapshot(path: str, cfg, state: np.ndarray, step: int, time: float, space: str) -> None:
    """One member's State (reference layout, complex128) as the reference's snapshot text."""
    nop = cfg.num_order_parameters
    nx, ny = cfg.nx, cfg.ny
    lines = []
    if space == "physical":
        phys = np.fft.irfft2(state, s=(ny, nx), axes=(-2, -1))
        lines.append("# snapshot space physical")
        lines.append(f"# step {step} time {_sci(time)}")
        lines.append(f"# nx {nx} ny {ny} order_parameters {nop}")
        lines.append("# x y rho" + "".join(f" psi_com{a}" for a in range(nop)) + " jx jy")
        order = [0] + [1 + a for a in range(nop)] + [nop + 1, nop + 2]
        cols = phys[order].reshape(len(order), -1)
        gy, gx = np.divmod(np.arange(nx * ny), nx)
        body = [f"{x} {y} " + " ".join(_sci(v) for v in cols[:, i]) for i, (x, y) in enumerate(zip(gx, gy))]
    elif space == "spectral":
        nkx = nx // 2 + 1
        lines.append("# snapshot space spectral")
        lines.append(f"# step {step} time {_sci(time)}")
        lines.append(f"# nkx {nkx} nky {ny} order_parameters {nop}")
        lines.append("# kx_index ky_index rho_real rho_imag" + "".join(f" psi_com{a}_real psi_com{a}_imag" for a in range(nop))
                     + " jx_real jx_imag jy_real jy_imag")
        flat = state.reshape(state.shape[0], -1)
        ky, kx = np.divmod(np.arange(nkx * ny), nkx)
        body = []
        for i, (x, y) in enumerate(zip(kx, ky)):
            vals = []
            for f in range(state.shape[0]):
                vals += [_sci(flat[f, i].real), _sci(flat[f, i].imag)]
            body.append(f"{x} {y} " + " ".join(vals))
    else:
        raise ValueError("snapshot space must be physical or spectral")
    with open(path, "w") as f:
        f.write("\n".join(lines + body) + "\n")


class Snapshot:
    """`measure <id> snapshot on nevery N file F space physical|spectral` over one engine member."""

    def __init__(self, engine, file: str, nevery: int, space: str, total_steps: int, member: int = 0):
        if space not in ("physical", "spectral"):
            raise ValueError("snapshot space must be physical or spectral")
        self.engine, self.file, self.nevery, self.space, self.total_steps, self.member = (
            engine, file, int(nevery), space, int(total_steps), member)

    def observe(self, step: int, time: float) -> None:
        if self.nevery <= 0 or step % self.nevery != 0:
            return
        path = snapshot_filename(self.file, step, self.total_steps)
        write_snapshot(path, self.engine.cfg, self.engine.get_state(self.member), step, time, self.space)

    def close(self) -> None:
        pass


class YokotaGreenKubo:
    """`measure <id> yokota_green_kubo on nevery N nblock B file F [mode diagonal|all]` over one
    engine member (measure_yokota_green_kubo.cc:16-225): the device accumulates the stress
    integrals (shhd_engine_gk_*); at every completed block the reference's table is rewritten,
    `nsample tau mode_index kx ky S_mean` per (tau, mode)."""

    def __init__(self, engine, file: str, nevery: int, nblock: int, mode: str = "diagonal", member: int = 0):
        if nevery <= 0:
            raise ValueError("yokota_green_kubo measure: nevery must be positive.")
        if nblock <= 0:
            raise ValueError("yokota_green_kubo measure: nblock must be positive.")
        if nblock % nevery != 0:
            raise ValueError("yokota_green_kubo measure: nblock must be divisible by nevery.")
        if mode not in ("diagonal", "all"):
            raise ValueError("yokota_green_kubo measure: mode must be diagonal|all.")
        self.engine, self.file, self.nevery, self.nblock, self.member = engine, file, int(nevery), int(nblock), member
        engine.gk_enable(self.nevery, self.nblock, mode)
        self.modes = list(engine.gk_modes)
        self.block_step = 0

    def observe(self, step: int, time: float) -> None:
        self.block_step += 1
        if self.block_step < self.nblock:
            return
        self.block_step = 0
        sums, nsample = self.engine.gk_read(self.member)
        cfg = self.engine.cfg
        lines = ["# nsample tau mode_index kx ky S_mean"]
        for ti in range(sums.shape[0]):
            tau = float((ti + 1) * self.nevery) * cfg.dt
            for mi, (nx, ny) in enumerate(self.modes):
                kx = 2.0 * 3.14159265358979323846 * float(nx) / cfg.lx
                ky = 2.0 * 3.14159265358979323846 * float(ny) / cfg.ly
                lines.append(f"{nsample} {_sci(tau)} {mi} {_sci(kx)} {_sci(ky)} {_sci(sums[ti, mi] / nsample)}")
        with open(self.file, "w") as f:
            f.write("\n".join(lines) + "\n")

    def close(self) -> None:
        pass


def parse_measures(engine, script_text: str, member: int = 0) -> List[object]:
    """The script's `measure` commands (time_series, snapshot, ave/profile, yokota_green_kubo) over one engine member."""
    total = sum(int(t[1]) for t in (ln.split("#", 1)[0].split() for ln in script_text.splitlines()) if len(t) >= 2 and t[0] == "run")
    out = []
    for raw in script_text.splitlines():
        t = raw.split("#", 1)[0].split()
        if len(t) < 4 or t[0] != "measure" or t[3] != "on":
            continue
        kind, rest = t[2], t[4:]
        kv, targets, i = {}, [], 0
        while i < len(rest):
            if rest[i] == "target":
                targets = rest[i + 1:]
                break
            kv[rest[i]] = rest[i + 1]
            i += 2
        if kind == "time_series":
            out.append(TimeSeries(engine, kv["file"], int(kv["nevery"]), targets, member))
        elif kind == "ave/profile":
            out.append(AveProfile(engine, kv["file"], kv["axis"], int(kv["nevery"]), int(kv["nblock"]), kv["average"], targets, member))
        elif kind == "snapshot":
            out.append(Snapshot(engine, kv["file"], int(kv["nevery"]), kv["space"], total, member))
        elif kind == "yokota_green_kubo":
            out.append(YokotaGreenKubo(engine, kv["file"], int(kv["nevery"]), int(kv["nblock"]), kv.get("mode", "diagonal"), member))
        else:
            raise NotImplementedError(f"measure style {kind}")
    return out


def run_script_measures(engine, script_text: str, member: int = 0) -> List[object]:
    """Advance `engine` through the script's `run` commands, observing its measures after each step.

    The engine steps in chunks that end on the next observed step; returns the closed measures.
    """
    measures = parse_measures(engine, script_text, member)
    runs = [int(t[1]) for t in (ln.split("#", 1)[0].split() for ln in script_text.splitlines()) if len(t) >= 2 and t[0] == "run"]
    step = int(engine.get_info().step_index)
    # ave/profile and yokota_green_kubo count every step they observe: step one at a time while one is present
    periods = [1] if any(isinstance(m, (AveProfile, YokotaGreenKubo)) for m in measures) else [m.nevery for m in measures]
    for n in runs:
        end = step + n
        while step < end:
            nxt = end
            for p in periods:
                nxt = min(nxt, (step // p + 1) * p)
            engine.step(nxt - step)
            step = nxt
            time = float(engine.get_info().time)   # advanced one dt per step, as the reference's driver
            for m in measures:
                m.observe(step, time)
    for m in measures:
        m.close()
    return measures


_PROFILE_FIELDS = {"rho": "rho", "jx": "jx", "jy": "jy", "vx": "vx", "vy": "vy"}
_PROFILE_FLUX = {"pi_xx": "pi_xx", "pixx": "pi_xx", "pi_xy": "pi_xy", "pixy": "pi_xy", "pi_yy": "pi_yy", "piyy": "pi_yy"}
_PROFILE_PSI = re.compile(r"^psi\[(\d+)\]$")
_PROFILE_JPSI = re.compile(r"^Jpsi\[(\d+)\]_[xy]$")


class AveProfile:
    """`measure <id> ave/profile on axis x|y nevery N nblock B file F average block|running target ...`
    over one engine member (measure_ave_profile.cc:180-453).

    Every nevery-th observed step adds a sample; every nblock-th step closes a block and writes
    the profiles averaged over the block (block) or over every block so far (running): the field
    averaged over the transverse axis on the padded grid, one bin per grid line.  Spectral
    targets (rho, psi[a], jx, jy; vx, vy = j / rho0 outside compressible dynamics) accumulate
    the one spectral line the transverse average needs, read from the device in FP64; the
    compressible vx, vy are summed over the transverse axis on the device per sample.  The flux
    targets (pi_xx pi_xy pi_yy, with the aliases pixx pixy piyy, and Jpsi[a]_x Jpsi[a]_y) read
    the last step's flux buffer along the same line from the engine's flux-line tap.
    """

    def __init__(self, engine, file: str, axis: str, nevery: int, nblock: int, average: str, targets: List[str], member: int = 0):
        cfg = engine.cfg
        if axis not in ("x", "y", "0", "1"):
            raise ValueError("ave/profile measure: axis must be x|y|0|1.")
        if average not in ("block", "running"):
            raise ValueError("ave/profile measure: average must be block|running.")
        if nevery <= 0:
            raise ValueError("ave/profile measure: nevery must be positive.")
        if nblock <= 0:
            raise ValueError("ave/profile measure: nblock must be positive.")
        self.axis = 0 if axis in ("x", "0") else 1
        self.engine, self.file, self.nevery, self.nblock, self.average, self.member = (
            engine, file, int(nevery), int(nblock), average, member)
        nop = cfg.num_order_parameters
        self.targets = []   # (name, kind, field index / component)
        for t in targets:
            if t in _PROFILE_FLUX:
                self.targets.append((_PROFILE_FLUX[t], "flux", _PROFILE_FLUX[t], None))
                continue
            j = _PROFILE_JPSI.match(t)
            if j:
                if not 0 <= int(j.group(1)) < nop:
                    raise ValueError(f"ave/profile target order-parameter index out of range: {t}")
                self.targets.append((t, "flux", t, None))
                continue
            m = _PROFILE_PSI.match(t)
            if m:
                a = int(m.group(1))
                if not 0 <= a < nop:
                    raise ValueError(f"ave/profile target order-parameter index out of range: {t}")
                self.targets.append((t, "spectral", 1 + a, 1.0))
            elif t in ("rho", "jx", "jy"):
                self.targets.append((t, "spectral", {"rho": 0, "jx": nop + 1, "jy": nop + 2}[t], 1.0))
            elif t in ("vx", "vy"):
                if cfg.mode == 2:
                    raise ValueError("AveProfileMeasure vx/vy is not available in quiescent dynamics.")
                comp = 0 if t == "vx" else 1
                if cfg.mode == 0:
                    self.targets.append((t, "velocity", comp, 1.0))
                else:
                    self.targets.append((t, "spectral_v", nop + 1 + comp, None))
            else:
                raise ValueError(f"unknown ave/profile target: {t}")
        self.nx, self.ny = cfg.nx, cfg.ny
        self.profile_size = self.nx if self.axis == 0 else self.ny
        self.spacing = (cfg.lx / cfg.nx) if self.axis == 0 else (cfg.ly / cfg.ny)
        self._rho0 = None
        self.block_step = 0
        self.samples_in_block = 0
        self.completed_blocks = 0
        self.running_samples = 0
        self._block = [None] * len(self.targets)
        self._running = [None] * len(self.targets)
        self._out: Optional[TextIO] = None
        if any(kind == "flux" for _n, kind, _i, _s in self.targets):
            # sampled every nevery-th observed step, counted from the step the measure starts at
            start = int(engine.get_info().step_index)
            engine.flux_line_enable(self.axis, every=self.nevery, phase=start)

    def _reference_density(self) -> float:
        """Re rho(0) / Ng of the first sample that needs it (measure_ave_profile.cc:123-149)."""
        if self._rho0 is None:
            line = self.engine.profile_line(0, 0, self.member)
            rho0 = line[0].real / (float(self.nx) * float(self.ny))
            if rho0 == 0.0:
                raise ValueError("AveProfileMeasure encountered zero reference density.")
            self._rho0 = rho0
        return self._rho0

    def _sample(self) -> None:
        flux = None
        for i, (_name, kind, idx, _scale) in enumerate(self.targets):
            if kind == "velocity":
                v = self.engine.profile_velocity(idx, self.axis, self.member)
            elif kind == "flux":
                if flux is None:
                    flux = self.engine.flux_line(self.axis, self.member)
                v = flux[idx]
            else:
                v = self.engine.profile_line(idx, self.axis, self.member)
                if kind == "spectral_v":
                    v = v * (1.0 / self._reference_density())
            self._block[i] = v.copy() if self._block[i] is None else self._block[i] + v
        self.samples_in_block += 1

    def _transverse_sum(self, kind: str, acc: np.ndarray) -> np.ndarray:
        """The field summed over the transverse axis from its accumulated line."""
        if kind == "velocity":
            return acc
        if self.axis == 0:
            row = np.zeros(self.nx // 2 + 1, dtype=np.complex128)
            row[:acc.size] = acc
            return np.fft.irfft(row, n=self.nx)
        col = np.zeros(self.ny, dtype=np.complex128)
        half = (acc.size + 1) // 2
        col[:half] = acc[:half]
        col[self.ny - (acc.size - half):] = acc[half:]
        return np.fft.ifft(col).real

    def _finish(self, step: int, time: float) -> None:
        if self.samples_in_block <= 0:
            raise RuntimeError("AveProfileMeasure tried to finish an empty block.")
        for i in range(len(self.targets)):
            self._running[i] = self._block[i].copy() if self._running[i] is None else self._running[i] + self._block[i]
        self.completed_blocks += 1
        self.running_samples += self.samples_in_block
        block = self.average == "block"
        src = self._block if block else self._running
        samples = self.samples_in_block if block else self.running_samples
        transverse = float(self.ny) if self.axis == 0 else float(self.nx)
        norm = float(samples) * transverse
        profiles = [self._transverse_sum(kind, acc) / norm for (_n, kind, _i, _s), acc in zip(self.targets, src)]
        lines = [f"# block {self.completed_blocks} step {step} time {_sci(time)} samples {samples}",
                 "# columns coord" + "".join(" " + n for n, _k, _i, _s in self.targets)]
        for b in range(self.profile_size):
            lines.append(_sci(self.spacing * float(b)) + "".join(" " + _sci(p[b]) for p in profiles))
        text = "\n".join(lines) + "\n\n"
        header = (f"# measure ave/profile\n# axis {'x' if self.axis == 0 else 'y'} nevery {self.nevery} nblock {self.nblock} "
                  f"average {self.average}\n")
        if block:
            if self._out is None:
                self._out = open(self.file, "w")
                self._out.write(header)
            self._out.write(text)
            self._out.flush()
        else:
            with open(self.file, "w") as f:
                f.write(header + text)
        self._block = [None] * len(self.targets)
        self.samples_in_block = 0

    def observe(self, step: int, time: float) -> None:
        self.block_step += 1
        if self.block_step % self.nevery == 0:
            self._sample()
        if self.block_step == self.nblock:
            self._finish(step, time)
            self.block_step = 0

    def close(self) -> None:
        if self._out is not None:
            self._out.close()
            self._out = None
