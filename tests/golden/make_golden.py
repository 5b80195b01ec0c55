"""Generate the golden fixtures from the reference's own code.

Runs in the build container, where the reference sources exist: it loads
oracle/_ref/libshhd_ref.so (the reference's src .cc files compiled against the
single-rank MPI / heFFTe shims, see oracle/Makefile) and records, per case:
the input script, the initial state the reference's initial-condition styles
produce, the deterministic RHS at that state, and two steps of the reference
integrator with the stochastic right-hand sides it drew.

    python tests/golden/make_golden.py            # writes tests/golden/ref_cases.npz
    python tests/golden/make_golden.py --initial  # writes tests/golden/ref_initial.npz
    python tests/golden/make_golden.py --measures # writes tests/golden/ref_measures.npz

The second form records, per initial-condition case, the reference's initial
state or, where the reference refuses the script, its error message.  The
third runs measure cases through the reference's own MeasurementManager and
records the state after every step, the noise each step drew and the text of
every file the measures wrote.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
from cases import CASES, FLUX_PROFILE_CASES, GK_CASES, IC_CASES, MEASURE_CASES, PROFILE_CASES  # noqa: E402

NSTEPS = 2


def main() -> None:
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so"))
    lib.shref_create.restype = ctypes.c_void_p
    lib.shref_last_error.restype = ctypes.c_char_p
    out = {}
    for name, script in CASES.items():
        h = ctypes.c_void_p(lib.shref_create(script.encode()))
        if not h.value:
            raise RuntimeError(f"{name}: {lib.shref_last_error().decode()}")
        info = (ctypes.c_long * 10)()
        dinfo = (ctypes.c_double * 4)()
        lib.shref_info(h, info, dinfo)
        nf, ny, hx = info[4], info[1], info[0] // 2 + 1
        shape = (nf, ny, hx)
        P = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        u0 = np.zeros(shape, complex)
        lib.shref_get_state(h, P(u0))
        det = np.zeros(shape, complex)
        assert lib.shref_rhs(h, ctypes.c_double(0.0), P(det)) == 0
        noise = np.zeros((NSTEPS, 2) + shape, complex)
        states = np.zeros((NSTEPS,) + shape, complex)
        for s in range(NSTEPS):
            rc = lib.shref_step(h, 1, P(noise[s]))
            if rc != 0:
                raise RuntimeError(f"{name}: {lib.shref_last_error().decode()}")
            lib.shref_get_state(h, P(states[s]))
        lib.shref_destroy(h)
        out[f"{name}/u0"] = u0
        out[f"{name}/det"] = det
        out[f"{name}/noise"] = noise
        out[f"{name}/states"] = states
        print(f"{name}: shape {shape}, |u0| {np.abs(u0).max():.3g}, |noise| {np.abs(noise).max():.3g}")
    np.savez_compressed(os.path.join(HERE, "ref_cases.npz"), **out)


def main_initial() -> None:
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so"))
    lib.shref_create.restype = ctypes.c_void_p
    lib.shref_last_error.restype = ctypes.c_char_p
    out = {}
    for name, script in IC_CASES.items():
        h = ctypes.c_void_p(lib.shref_create(script.encode()))
        if not h.value:
            out[f"{name}/error"] = np.array(lib.shref_last_error().decode())
            print(f"{name}: error {out[name + '/error']}")
            continue
        info = (ctypes.c_long * 10)()
        dinfo = (ctypes.c_double * 4)()
        lib.shref_info(h, info, dinfo)
        u0 = np.zeros((info[4], info[1], info[0] // 2 + 1), complex)
        lib.shref_get_state(h, u0.ctypes.data_as(ctypes.c_void_p))
        lib.shref_destroy(h)
        out[f"{name}/u0"] = u0
        print(f"{name}: shape {u0.shape}, |u0| {np.abs(u0).max():.3g}")
    np.savez_compressed(os.path.join(HERE, "ref_initial.npz"), **out)


def main_measures() -> None:
    import tempfile
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libshhd_ref.so"))
    lib.shref_create.restype = ctypes.c_void_p
    lib.shref_last_error.restype = ctypes.c_char_p
    out = {}
    for name, template in {**MEASURE_CASES, **PROFILE_CASES, **FLUX_PROFILE_CASES, **GK_CASES}.items():
        with tempfile.TemporaryDirectory() as tmp:
            script = template.replace("@DIR@", tmp)
            nsteps = int(script.rsplit("run ", 1)[1].split()[0])
            h = ctypes.c_void_p(lib.shref_create(script.encode()))
            if not h.value:
                raise RuntimeError(f"{name}: {lib.shref_last_error().decode()}")
            info = (ctypes.c_long * 10)()
            dinfo = (ctypes.c_double * 4)()
            lib.shref_info(h, info, dinfo)
            shape = (info[4], info[1], info[0] // 2 + 1)
            u0 = np.zeros(shape, complex)
            lib.shref_get_state(h, u0.ctypes.data_as(ctypes.c_void_p))
            states = np.zeros((nsteps,) + shape, complex)
            noise = np.zeros((nsteps, 2) + shape, complex)
            for s in range(nsteps):
                if lib.shref_step(h, 1, noise[s].ctypes.data_as(ctypes.c_void_p)) != 0:
                    raise RuntimeError(f"{name}: {lib.shref_last_error().decode()}")
                lib.shref_get_state(h, states[s].ctypes.data_as(ctypes.c_void_p))
            lib.shref_finalize(h)
            lib.shref_destroy(h)
            out[f"{name}/u0"] = u0
            out[f"{name}/states"] = states
            out[f"{name}/noise"] = noise
            for fn in sorted(os.listdir(tmp)):
                with open(os.path.join(tmp, fn)) as f:
                    out[f"{name}/file/{fn}"] = np.array(f.read())
            print(f"{name}: {nsteps} steps, files {sorted(os.listdir(tmp))}")
    np.savez_compressed(os.path.join(HERE, "ref_measures.npz"), **out)


if __name__ == "__main__":
    if "--initial" in sys.argv[1:]:
        main_initial()
    elif "--measures" in sys.argv[1:]:
        main_measures()
    else:
        main()
