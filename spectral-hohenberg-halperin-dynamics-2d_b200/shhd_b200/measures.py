"""The reference's `measure` commands over an engine, written in the reference's file formats.

  time_series (measure_time_series.cc:109-286): the energy columns E_T E_K E_psi E_C
      (shhd_engine_energies) and the spectral L2 columns |rho|^2 ... |d_psi[a]|^2
      (shhd_engine_l2_sums), FP64 sums on the device; one line per observed step,
      `step time v...` in scientific notation with 16 digits.  The k = 0 flux
      columns pi_xx pi_xy pi_yy Jpsi[a]_x Jpsi[a]_y come from the engine's flux
      tap (shhd_engine_flux0_*), enabled when a column asks for it: the last
      step's stage-weighted (0, 0) fluxes, as the reference's flux buffer holds.
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
            engine.flux0_enable()
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


def parse_measures(engine, script_text: str, member: int = 0) -> List[object]:
    """The script's `measure` commands (time_series, snapshot) over one engine member."""
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
        elif kind == "snapshot":
            out.append(Snapshot(engine, kv["file"], int(kv["nevery"]), kv["space"], total, member))
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
    periods = [m.nevery for m in measures if m.nevery > 0]
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
