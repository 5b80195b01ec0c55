"""Binary restart files in the reference's State layout.

The reference accepts `restart on file <name>` (param_parser.cc:493-511) but
writes nothing; this module is the missing writer and reader.  A file holds
everything a run needs to continue bit-for-bit in FP64:

    magic    8 bytes  b"SHHDRST1"
    header   int64 x 8: nfields, nx, ny, batch, step_index, config bytes, reserved x 2
             float64:   time
    config   the shhd_config struct as the engine was created with it
    states   batch x nfields x ny x (nx/2 + 1) complex128, little endian

The step index keys the noise (Philox counter), so an engine loaded from the
file draws the same noise the uninterrupted run would have drawn.
"""
from __future__ import annotations

import ctypes
import struct
from typing import List, Tuple

import numpy as np

from . import Config, Engine

MAGIC = b"SHHDRST1"
_HEADER = struct.Struct("<8q d")


def write_restart(path: str, cfg: Config, states: List[np.ndarray], step_index: int, time: float) -> None:
    """Write `states` (one reference-layout complex128 array per member)."""
    if not states:
        raise ValueError("no state to write")
    shape = states[0].shape
    for s in states:
        if s.shape != shape:
            raise ValueError("all members must have the same state shape")
    raw = bytes(memoryview(cfg).cast("B"))
    nfields, ny, hx = shape
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(_HEADER.pack(nfields, cfg.nx, cfg.ny, len(states), int(step_index), len(raw), 0, 0, float(time)))
        f.write(raw)
        for s in states:
            f.write(np.ascontiguousarray(s, dtype="<c16").tobytes())


def read_restart(path: str) -> Tuple[Config, List[np.ndarray], int, float]:
    """(configuration, member states, step index, time) of a restart file."""
    with open(path, "rb") as f:
        if f.read(len(MAGIC)) != MAGIC:
            raise ValueError(f"{path}: not a restart file")
        nfields, nx, ny, batch, step_index, nraw, _r0, _r1, time = _HEADER.unpack(f.read(_HEADER.size))
        raw = f.read(nraw)
        if nraw != ctypes.sizeof(Config) or len(raw) != nraw:
            raise ValueError(f"{path}: configuration block of {nraw} bytes, expected {ctypes.sizeof(Config)}")
        cfg = Config()
        ctypes.memmove(ctypes.byref(cfg), raw, nraw)
        if (cfg.nx, cfg.ny) != (nx, ny):
            raise ValueError(f"{path}: header grid does not match the configuration")
        n = nfields * ny * (nx // 2 + 1)
        states = []
        for _ in range(batch):
            buf = f.read(16 * n)
            if len(buf) != 16 * n:
                raise ValueError(f"{path}: truncated state data")
            states.append(np.frombuffer(buf, dtype="<c16").reshape(nfields, ny, nx // 2 + 1).copy())
    return cfg, states, int(step_index), float(time)


def save_engine(path: str, engine: Engine) -> None:
    """Every member's state, the step index and the time of `engine`."""
    info = engine.get_info()
    write_restart(path, engine.cfg, [engine.get_state(m) for m in range(engine.cfg.batch)], info.step_index, info.time)


def load_engine(path: str, precision: int = None) -> Engine:
    """A new engine continuing the run saved in `path` (optionally at another precision)."""
    cfg, states, step_index, time = read_restart(path)
    if precision is not None:
        cfg.precision = precision
    engine = Engine(cfg)
    for m, s in enumerate(states):
        engine.set_state(s, member=m)
    engine.set_time(step_index, time)
    return engine
