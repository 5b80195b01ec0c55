"""Time-series energy / L2 columns and snapshot files against the reference's own measure output.

The fixtures (tests/golden/ref_measures.npz, made by make_golden.py --measures)
hold, per case, the state after every step, the noise each step drew and the
files the reference's MeasurementManager wrote along that trajectory.

CPU: the oracle's restatement of the energy, L2 and k = 0 flux columns
reproduces the reference's time-series values (1e-12 relative; the flux
columns on the scale of their terms, which can cancel); the snapshot writer
reproduces the reference's snapshot files (the spectral file byte for byte,
the physical one to 1e-12 of the field's scale: the host inverse transform is
not the reference's); snapshot file names and the column checks.

GPU: the engine's FP64 device sums reproduce the reference's values on the
reference's states (FP64 1e-12, FP32 1e-5 relative); replaying the
reference's noise, the flux tap reproduces the reference's k = 0 flux
columns step by step, and the measures written along the engine's own
trajectory reproduce the reference's files (every column).
"""
import os

import numpy as np
import pytest

import shhd_oracle as so
from golden.cases import MEASURE_CASES

DATA = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_measures.npz"))
ENERGY = ("E_T", "E_K", "E_psi", "E_C")


def _ts(name):
    """(columns, rows) of the reference's ts.dat: rows are (step, time, {column: value})."""
    lines = str(DATA[f"{name}/file/ts.dat"]).splitlines()
    cols = lines[1].split()[3:]
    rows = []
    for ln in lines[2:]:
        t = ln.split()
        rows.append((int(t[0]), float(t[1]), dict(zip(cols, map(float, t[2:])))))
    return cols, rows


def _close(got, want, rtol, scale=None):
    s = scale if scale is not None else max(abs(want), 1e-300)
    return abs(got - want) <= rtol * s


def _script(name, tmp):
    return MEASURE_CASES[name].replace("@DIR@", str(tmp))


@pytest.mark.parametrize("name", sorted(MEASURE_CASES))
def test_oracle_columns_match_reference_measure(name, tmp_path):
    cfg = so.parse_script(_script(name, tmp_path))
    cols, rows = _ts(name)
    states = DATA[f"{name}/states"]
    for s, (step, _time, want) in enumerate(rows):
        got = {**so.time_series_energies(cfg, states[s]), **so.time_series_l2(cfg, states[s])}
        for c in cols:
            if c in got:
                # E_T sums terms of either sign: compare on the scale of its largest term
                scale = max(abs(want["E_K"]), abs(want["E_psi"]), abs(want["E_C"])) if c == "E_T" else None
                assert _close(got[c], want[c], 1e-12, scale), (name, step, c, got[c], want[c])


def _compare_snapshot(text, want_text, exact):
    got, want = text.splitlines(), want_text.splitlines()
    assert len(got) == len(want)
    assert got[:4] == want[:4]                       # the four header lines
    if exact:
        assert text == want_text
        return
    g = np.array([[float(x) for x in ln.split()] for ln in got[4:]])
    w = np.array([[float(x) for x in ln.split()] for ln in want[4:]])
    assert np.array_equal(g[:, :2], w[:, :2])        # grid indices
    scale = np.max(np.abs(w[:, 2:]), axis=0)
    assert np.all(np.abs(g[:, 2:] - w[:, 2:]) <= 1e-12 * scale)


@pytest.mark.parametrize("name", sorted(MEASURE_CASES))
def test_snapshot_writer_matches_reference_files(name, tmp_path):
    import shhd_b200 as sb
    from shhd_b200.measures import snapshot_filename, write_snapshot
    text = _script(name, tmp_path)
    cfg = sb.config_from_script(text)
    nsteps = DATA[f"{name}/states"].shape[0]
    state = DATA[f"{name}/states"][nsteps - 1]
    _cols, rows = _ts(name)
    step, time = rows[-1][0], rows[-1][1]
    for space, prefix in (("physical", "phys"), ("spectral", "spec")):
        path = snapshot_filename(str(tmp_path / prefix), step, nsteps)
        write_snapshot(path, cfg, state, step, time, space)
        fn = os.path.basename(path)
        assert f"{name}/file/{fn}" in DATA.files, fn
        with open(path) as f:
            _compare_snapshot(f.read(), str(DATA[f"{name}/file/{fn}"]), exact=(space == "spectral"))


def test_snapshot_filename_width():
    from shhd_b200.measures import snapshot_filename
    assert snapshot_filename("a", 3, 3) == "a_step03.snapshot"
    assert snapshot_filename("a", 50, 1000) == "a_step00050.snapshot"
    assert snapshot_filename("a", 0, 0) == "a_step00.snapshot"


def _flux_scale(want, c):
    """Scale of a k = 0 flux column: its terms (pressure, advection) can cancel."""
    if c.startswith("pi_"):
        return max(abs(want["pi_xx"]), abs(want["pi_yy"]), abs(want[c]), 1e-300)
    return max(max(abs(v) for k, v in want.items() if k.startswith("Jpsi")), 1e-300)


@pytest.mark.parametrize("name", sorted(MEASURE_CASES))
def test_oracle_k0_flux_matches_reference_measure(name, tmp_path):
    cfg = so.parse_script(_script(name, tmp_path))
    cols, rows = _ts(name)
    o = so.Oracle(cfg)
    u = DATA[f"{name}/u0"]
    for s, (step, _time, want) in enumerate(rows):
        nz = DATA[f"{name}/noise"][s]
        _u, got = o.step_with_k0_flux(u, (nz[0], nz[1]) if cfg.integrator == "srk3" else (nz[0],))
        for c in cols:
            if c in got:
                assert _close(got[c], want[c], 1e-12, _flux_scale(want, c)), (name, step, c, got[c], want[c])
        u = DATA[f"{name}/states"][s]


def test_time_series_rejects_unknown_columns():
    from shhd_b200.measures import TimeSeries

    class _Eng:
        class cfg:
            num_order_parameters = 1

    with pytest.raises(ValueError):
        TimeSeries(_Eng(), "x", 1, ["Jpsi[1]_x"])
    with pytest.raises(ValueError):
        TimeSeries(_Eng(), "x", 1, ["|psi[1]|^2"])
    with pytest.raises(ValueError):
        TimeSeries(_Eng(), "x", 1, ["E_Q"])
    with pytest.raises(ValueError):
        TimeSeries(_Eng(), "x", 0, ["E_K"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(MEASURE_CASES))
def test_device_columns_match_reference_measure(name, precision, tmp_path):
    import shhd_b200 as sb
    cfg = sb.config_from_script(_script(name, tmp_path))
    cfg.precision = precision
    rtol = 1e-12 if precision == 0 else 1e-5
    cols, rows = _ts(name)
    states = DATA[f"{name}/states"]
    with sb.Engine(cfg) as eng:
        for s, (step, _time, want) in enumerate(rows):
            eng.set_state(states[s])
            got = {**eng.time_series_energies(), **eng.time_series_l2()}
            for c in cols:
                if c in got:
                    scale = max(abs(want["E_K"]), abs(want["E_psi"]), abs(want["E_C"])) if c == "E_T" else None
                    assert _close(got[c], want[c], rtol, scale), (name, precision, step, c, got[c], want[c])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(MEASURE_CASES))
def test_device_k0_flux_matches_reference_measure(name, precision, tmp_path):
    """Replaying the reference's noise, the flux tap reads the reference's pi_* / Jpsi columns."""
    import shhd_b200 as sb
    cfg = sb.config_from_script(_script(name, tmp_path))
    cfg.precision = precision
    cfg.noise_source = 1
    rtol = 1e-11 if precision == 0 else 2e-5
    cols, rows = _ts(name)
    noise = DATA[f"{name}/noise"]
    with sb.Engine(cfg) as eng:
        eng.set_state(DATA[f"{name}/u0"])
        eng.flux0_enable()
        for s, (step, _time, want) in enumerate(rows):
            eng.set_external_noise(noise[s, 0], noise[s, 1])
            eng.step(1)
            got = eng.flux0_read()
            for c in cols:
                if c in got:
                    assert _close(got[c], want[c], rtol, _flux_scale(want, c)), (name, precision, step, c, got[c], want[c])


@pytest.mark.gpu
def test_k0_flux_survives_graph_replay(tmp_path):
    """The tap is part of captured steps: graph replays record the same last-step flux."""
    import shhd_b200 as sb
    name = "srk3_compressible_n2"
    cfg = sb.config_from_script(_script(name, tmp_path))
    with sb.Engine(cfg) as g, sb.Engine(cfg) as d:
        for e in (g, d):
            e.set_state(DATA[f"{name}/u0"])
            e.flux0_enable()
        g.set_graph_chunk(4)
        g.step(8)
        d.step(4)
        d.step(4)
        assert g.flux0_read() == d.flux0_read()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["srk3_compressible_n2", "srk3_incompressible_n1_forces", "euler_quiescent_n2_quadratic"])
def test_measure_files_along_the_reference_trajectory(name, tmp_path):
    """Replaying the reference's noise, the engine's measures write the reference's files."""
    import shhd_b200 as sb
    from shhd_b200.measures import Snapshot, TimeSeries
    text = _script(name, tmp_path)
    cfg = sb.config_from_script(text)
    cfg.noise_source = 1
    cols, rows = _ts(name)
    nsteps = DATA[f"{name}/states"].shape[0]
    noise = DATA[f"{name}/noise"]
    with sb.Engine(cfg) as eng:
        eng.set_state(DATA[f"{name}/u0"])
        ts = TimeSeries(eng, str(tmp_path / "ts_dev.dat"), 1, cols)
        snaps = [Snapshot(eng, str(tmp_path / "phys"), 3, "physical", nsteps), Snapshot(eng, str(tmp_path / "spec"), 3, "spectral", nsteps)]
        for s in range(nsteps):
            eng.set_external_noise(noise[s, 0], noise[s, 1])
            eng.step(1)
            info = eng.get_info()
            for m in [ts] + snaps:
                m.observe(int(info.step_index), float(info.time))
        ts.close()
    with open(tmp_path / "ts_dev.dat") as f:
        lines = f.read().splitlines()
    assert lines[0] == "# measure time_series"
    assert lines[1] == str(DATA[f"{name}/file/ts.dat"]).splitlines()[1]
    for ln, (step, time, want) in zip(lines[2:], rows):
        t = ln.split()
        assert int(t[0]) == step and t[1] == f"{time:.16e}"
        for c, v in zip(cols, map(float, t[2:])):
            if c.startswith("pi_") or c.startswith("Jpsi"):
                scale = _flux_scale(want, c)
            else:
                scale = max(abs(want["E_K"]), abs(want["E_psi"]), abs(want["E_C"])) if c == "E_T" else None
            assert _close(v, want[c], 1e-11, scale), (name, step, c, v, want[c])
    for prefix in ("phys", "spec"):
        fn = f"{prefix}_step03.snapshot"
        with open(tmp_path / fn) as f:
            # the engine's trajectory differs from the reference's in the last digits
            _compare_snapshot(f.read(), str(DATA[f"{name}/file/{fn}"]), exact=False)


@pytest.mark.gpu
@pytest.mark.parametrize("te", ["euler/incompressible", "euler/quiescent"])
def test_fp32_static_fields_keep_their_k0_values_through_euler_swaps(te):
    """Euler engines swap their state buffers every step; the FP64 k = 0 copies of the fields a
    mode does not evolve (density, and momentum in quiescent dynamics) must follow, since the
    measures read them: density line, reference density and energies after an odd step count."""
    import shhd_b200 as sb
    from helpers import random_state, script
    text = script(grid=(32, 32), length=(64.0, 64.0), nop=1, dt=0.01, te=te, cT=None, eta=0.05 if "incomp" in te else 0.0,
                  zeta=0.0, nonlinear="momentum" if "incomp" in te else None)
    ocfg = so.parse_script(text)
    u0 = random_state(ocfg, seed=4, rho0=1.3, transverse=True)
    got = {}
    for precision in (0, 1):
        cfg = sb.config_from_script(text)
        cfg.precision = precision
        with sb.Engine(cfg) as eng:
            eng.set_state(u0)
            eng.step(3)
            got[precision] = (eng.profile_line(0, 0), eng.time_series_energies())
    assert got[1][0][0] == got[0][0][0] == u0[0, 0, 0]
    for k in ENERGY:
        assert _close(got[1][1][k], got[0][1][k], 1e-5, max(abs(v) for v in got[0][1].values())), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_measures_of_batched_members_equal_single_engines(precision):
    """Every device measure reads its own member of a batched engine (the served-slot case)."""
    import shhd_b200 as sb
    from helpers import random_state, script
    text = script(grid=(32, 32), length=(64.0, 64.0), nop=2, dt=0.01, noise=None)
    ocfg = so.parse_script(text)
    states = [random_state(ocfg, seed=s, rho0=1.0 + 0.1 * s) for s in (3, 8)]

    def measure(eng, m):
        return (eng.time_series_energies(m), eng.time_series_l2(m), eng.flux0_read(m), eng.profile_line(1, 0, m),
                eng.profile_line(0, 1, m), eng.profile_velocity(1, 0, m), eng.flux_line(1, m))

    def engine(batch):
        cfg = sb.config_from_script(text)
        cfg.precision = precision
        cfg.batch = batch
        e = sb.Engine(cfg)
        e.flux0_enable()
        e.flux_line_enable(1)
        return e

    with engine(2) as both:
        for m, st in enumerate(states):
            both.set_state(st, member=m)
        both.step(2)
        got = [measure(both, m) for m in range(2)]
    for m, st in enumerate(states):
        with engine(1) as one:
            one.set_state(st)
            one.step(2)
            want = measure(one, 0)
        for g, w in zip(got[m], want):
            if isinstance(w, dict):
                for k in w:
                    assert np.allclose(g[k], w[k], rtol=1e-12, atol=0.0), (m, k)
            else:
                assert np.allclose(g, w, rtol=1e-12, atol=1e-300), m


@pytest.mark.gpu
def test_scheduled_flux_taps_record_the_sampled_steps():
    """A tap asked for every n-th step records, on those steps, what an always-on tap records
    (direct launches and graph replays alike); requests from two measures merge to their gcd."""
    import shhd_b200 as sb
    from helpers import random_state, script
    text = script(grid=(32, 32), length=(64.0, 64.0), nop=1, dt=0.01, noise="kBT 0.002 seed 4")
    u0 = random_state(so.parse_script(text), seed=6)
    cfg = sb.config_from_script(text)
    with sb.Engine(cfg) as every, sb.Engine(cfg) as sched:
        for e in (every, sched):
            e.set_state(u0)
        every.flux0_enable()
        every.flux_line_enable(1)
        sched.flux0_enable(every=3)
        sched.flux_line_enable(1, every=4, phase=2)
        sched.set_graph_chunk(2)
        for step in range(1, 11):
            every.step(1)
            sched.step(1)
            if step % 3 == 0:
                assert sched.flux0_read() == every.flux0_read(), step
            if step % 4 == 2:
                a, b = sched.flux_line(1), every.flux_line(1)
                assert all(np.array_equal(a[k], b[k]) for k in a), step
        sched.flux_tap_request(0, 2, 0)      # merged with every=3, phase 0: every step
        assert sched._tap_schedules[0] == (1, 0)
