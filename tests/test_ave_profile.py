"""ave/profile against the reference's own profile files (tests/golden/ref_measures.npz).

CPU: AveProfile's block / running bookkeeping, spectral-line transverse sums
and file format, fed by a numpy stand-in for the engine's two per-sample calls
(profile_line: the ky = 0 row or kx = 0 column of a field; profile_velocity:
the compressible j / rho summed over the transverse axis) on the reference's
states, reproduce the reference's files: the header and block lines exactly,
the values to 1e-12 of each column's scale (floored at round-off of the
largest column: a profile that vanishes analytically holds the reference's
transform round-off).

Flux targets: the reference's flux buffer holds noise draws the engine cannot
reconstruct from a replayed divergence, so the flux-profile fixtures are
noise-free runs; the oracle's flux-buffer restatement and the engine's
flux-line tap both write the reference's files there, and with the engine's
own noise the tap equals the oracle's flux buffer (noise flux and projection
pressure included).

GPU: the engine, replaying the reference's noise, writes the same files
(values to 1e-11 of each column's scale); FP32 engines to 1e-5.
"""
import os

import numpy as np
import pytest

import shhd_oracle as so
from golden.cases import FLUX_PROFILE_CASES, PROFILE_CASES

DATA = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_measures.npz"))


class _HostEngine:
    """The engine's profile calls restated on a reference-layout state (numpy)."""

    def __init__(self, cfg):
        self.cfg = cfg
        self.state = None
        self.flux = None          # the last step's flux buffer (oracle fields)

    def _line(self, field2d, axis):
        c = self.cfg
        if axis == 0:
            return field2d[0, :c.active_nx // 2].copy()
        half = c.active_ny // 2
        ky = np.concatenate([np.arange(half), np.arange(-(half - 1), 0)])
        return field2d[ky % c.ny, 0].copy()

    def flux_line_enable(self, axis, every=1, phase=0):
        pass

    def get_info(self):
        class _Info:
            step_index = 0
        return _Info()

    def flux_line(self, axis, member=0):
        return {k: self._line(v, axis) for k, v in self.flux.items()}

    def profile_line(self, field, axis, member=0):
        c = self.cfg
        if axis == 0:
            return self.state[field, 0, :c.active_nx // 2].copy()
        half = c.active_ny // 2
        ky = np.concatenate([np.arange(half), np.arange(-(half - 1), 0)])
        return self.state[field, ky % c.ny, 0].copy()

    def profile_velocity(self, component, axis, member=0):
        c = self.cfg
        n = c.num_order_parameters
        rho = np.fft.irfft2(self.state[0], s=(c.ny, c.nx))
        j = np.fft.irfft2(self.state[n + 1 + component], s=(c.ny, c.nx))
        v = j / rho
        return v.sum(axis=0) if axis == 0 else v.sum(axis=1)


def _compare_profile_files(got_text, want_text, rtol):
    got, want = got_text.splitlines(), want_text.splitlines()
    assert len(got) == len(want)
    cols = None
    for g, w in zip(got, want):
        if w.startswith("#") or not w.strip():
            assert g == w
            continue
        gv = np.array([float(x) for x in g.split()])
        wv = np.array([float(x) for x in w.split()])
        assert gv.shape == wv.shape
        cols = wv if cols is None else cols
        assert abs(gv[0] - wv[0]) <= 1e-15 * max(abs(wv[0]), 1.0)
    # values: per block, per column, on the column's scale
    blocks_g = [b for b in got_text.split("\n\n") if b.strip()]
    blocks_w = [b for b in want_text.split("\n\n") if b.strip()]
    for bg, bw in zip(blocks_g, blocks_w):
        rg = np.array([[float(x) for x in ln.split()] for ln in bg.splitlines() if ln and not ln.startswith("#")])
        rw = np.array([[float(x) for x in ln.split()] for ln in bw.splitlines() if ln and not ln.startswith("#")])
        scale = np.max(np.abs(rw[:, 1:]), axis=0)
        # a profile that vanishes analytically (e.g. incompressible jx over x) holds the
        # reference's transform round-off: floor the scale at round-off of the largest column
        floor = 1e-15 / rtol * np.max(scale)
        assert np.all(np.abs(rg[:, 1:] - rw[:, 1:]) <= rtol * np.maximum(scale, floor)), (rg[:, 1:] - rw[:, 1:]).max()


def _script(name, tmp):
    return PROFILE_CASES[name].replace("@DIR@", str(tmp))


def _files(name):
    pre = f"{name}/file/"
    return {k[len(pre):]: str(DATA[k]) for k in DATA.files if k.startswith(pre)}


@pytest.mark.parametrize("name", sorted(PROFILE_CASES))
def test_profile_bookkeeping_matches_reference_files(name, tmp_path):
    import shhd_b200 as sb
    from shhd_b200.measures import AveProfile, parse_measures
    text = _script(name, tmp_path)
    cfg = sb.config_from_script(text)
    eng = _HostEngine(cfg)
    measures = parse_measures(eng, text)
    assert all(isinstance(m, AveProfile) for m in measures)
    states = DATA[f"{name}/states"]
    time = 0.0
    for s in range(states.shape[0]):
        eng.state = states[s]
        time += cfg.dt
        for m in measures:
            m.observe(s + 1, time)
    for m in measures:
        m.close()
    for fn, want in _files(name).items():
        with open(tmp_path / fn) as f:
            _compare_profile_files(f.read(), want, 1e-12)


@pytest.mark.parametrize("name", sorted(FLUX_PROFILE_CASES))
def test_flux_profiles_from_the_oracle_match_reference_files(name, tmp_path):
    """The oracle's flux-buffer restatement (noise-free steps) through AveProfile writes the
    reference's flux-profile files."""
    import shhd_b200 as sb
    from shhd_b200.measures import parse_measures
    text = FLUX_PROFILE_CASES[name].replace("@DIR@", str(tmp_path))
    cfg = sb.config_from_script(text)
    o = so.Oracle(so.parse_script(text))
    eng = _HostEngine(cfg)
    measures = parse_measures(eng, text)
    states = DATA[f"{name}/states"]
    u = DATA[f"{name}/u0"]
    time = 0.0
    for s in range(states.shape[0]):
        u_next, eng.flux = o.step_with_flux_fields(u, None)
        assert so.rel_l2(u_next, states[s]) < 1e-12
        u = eng.state = states[s]
        time += cfg.dt
        for m in measures:
            m.observe(s + 1, time)
    for m in measures:
        m.close()
    pre = f"{name}/file/"
    for k in DATA.files:
        if k.startswith(pre):
            with open(tmp_path / k[len(pre):]) as f:
                _compare_profile_files(f.read(), str(DATA[k]), 1e-11)


def test_profile_rejects_what_the_reference_rejects(tmp_path):
    import shhd_b200 as sb
    from shhd_b200.measures import AveProfile
    text = _script("profile_euler_quiescent_n2_quadratic", tmp_path)
    eng = _HostEngine(sb.config_from_script(text))
    with pytest.raises(ValueError, match="not available in quiescent"):
        AveProfile(eng, "f", "x", 1, 1, "block", ["vx"])
    with pytest.raises(ValueError, match="index out of range"):
        AveProfile(eng, "f", "x", 1, 1, "block", ["psi[2]"])
    with pytest.raises(ValueError, match="axis must be"):
        AveProfile(eng, "f", "z", 1, 1, "block", ["rho"])
    with pytest.raises(ValueError, match="average must be"):
        AveProfile(eng, "f", "x", 1, 1, "mean", ["rho"])
    with pytest.raises(ValueError, match="unknown ave/profile target"):
        AveProfile(eng, "f", "x", 1, 1, "block", ["temperature"])
    with pytest.raises(ValueError, match="index out of range"):
        AveProfile(eng, "f", "y", 1, 1, "block", ["Jpsi[2]_x"])


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(FLUX_PROFILE_CASES))
def test_device_flux_profiles_match_reference_files(name, precision, tmp_path):
    """Noise-free runs: the engine's flux-line tap through AveProfile writes the reference's files."""
    import shhd_b200 as sb
    from shhd_b200.measures import run_script_measures
    text = FLUX_PROFILE_CASES[name].replace("@DIR@", str(tmp_path))
    cfg = sb.config_from_script(text)
    cfg.precision = precision
    with sb.Engine(cfg) as eng:
        eng.set_state(DATA[f"{name}/u0"])
        run_script_measures(eng, text)
        assert so.rel_l2(eng.get_state(), DATA[f"{name}/states"][-1]) < (1e-12 if precision == 0 else 1e-5)
    pre = f"{name}/file/"
    for k in DATA.files:
        if k.startswith(pre):
            with open(tmp_path / k[len(pre):]) as f:
                _compare_profile_files(f.read(), str(DATA[k]), 1e-10 if precision == 0 else 1e-4)


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [0, 1])
@pytest.mark.parametrize("te", ["srk3/compressible", "srk3/incompressible", "euler/compressible"])
def test_device_flux_line_with_noise_matches_the_oracle(te, axis):
    """With the engine's own (Philox) noise, the flux line equals the oracle's flux buffer:
    deterministic stage fluxes, the first draw's noise flux / sqrt(dt), the projection pressure."""
    import shhd_b200 as sb
    from helpers import random_state, script
    incomp = "incompressible" in te
    text = script(grid=(32, 32), length=(64.0, 64.0), nop=2, dt=0.01, te=te, cT=None if incomp else 1.0, eta=0.3, zeta=0.0 if incomp else 0.7,
                  nonlinear="all", noise="kBT 0.002 seed 9")
    ocfg = so.parse_script(text)
    u0 = random_state(ocfg, seed=13, transverse=incomp)
    o = so.Oracle(ocfg)
    cfg = sb.config_from_script(text)
    with sb.Engine(cfg) as eng:
        eng.set_state(u0)
        eng.flux_line_enable(axis)
        u = u0
        for _ in range(2):
            u, want = o.step_with_flux_fields(u, "philox")
            eng.step(1)
            got = eng.flux_line(axis)
            h = _HostEngine(cfg)
            for k, v in want.items():
                w = h._line(v, axis)
                assert np.max(np.abs(got[k] - w)) <= 1e-10 * max(np.max(np.abs(w)), 1e-300), k


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(PROFILE_CASES))
def test_device_profiles_match_reference_files(name, precision, tmp_path):
    import shhd_b200 as sb
    from shhd_b200.measures import parse_measures
    text = _script(name, tmp_path)
    cfg = sb.config_from_script(text)
    cfg.precision = precision
    cfg.noise_source = 1
    noise = DATA[f"{name}/noise"]
    with sb.Engine(cfg) as eng:
        eng.set_state(DATA[f"{name}/u0"])
        measures = parse_measures(eng, text)
        for s in range(noise.shape[0]):
            eng.set_external_noise(noise[s, 0], noise[s, 1])
            eng.step(1)
            info = eng.get_info()
            for m in measures:
                m.observe(int(info.step_index), float(info.time))
        for m in measures:
            m.close()
    for fn, want in _files(name).items():
        with open(tmp_path / fn) as f:
            _compare_profile_files(f.read(), want, 1e-11 if precision == 0 else 1e-5)
