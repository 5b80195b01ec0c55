"""The Yokota-Green-Kubo measure's file against the reference's own (tests/golden/ref_measures.npz).

With eta = zeta = 0 the momentum carries no noise and psi does not enter its
equations, so pi_xy and every S_mean are deterministic although `fix noise`
is on (the measure needs its kBT): the reference's table can be reproduced
exactly, by the oracle (CPU) and by the engine with its own noise draws for
psi (GPU).  Integer columns and wave numbers must match as text, S_mean to
1e-10 relative.
"""
import os

import numpy as np
import pytest

import shhd_oracle as so
from golden.cases import GK_CASES

DATA = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_measures.npz"))


def _compare_gk(got_text, want_text, rtol):
    got, want = got_text.splitlines(), want_text.splitlines()
    assert got[0] == want[0] == "# nsample tau mode_index kx ky S_mean"
    assert len(got) == len(want)
    for g, w in zip(got[1:], want[1:]):
        gt, wt = g.split(), w.split()
        assert gt[:5] == wt[:5], (g, w)
        assert abs(float(gt[5]) - float(wt[5])) <= rtol * abs(float(wt[5])), (g, w)


def _gk_line(text):
    for ln in text.splitlines():
        t = ln.split()
        if t and t[0] == "measure" and t[2] == "yokota_green_kubo":
            kv = dict(zip(t[4::2], t[5::2]))
            return int(kv["nevery"]), int(kv["nblock"]), os.path.basename(kv["file"]), kv.get("mode", "diagonal")
    raise AssertionError("no yokota_green_kubo line")


@pytest.mark.parametrize("name", sorted(GK_CASES))
def test_oracle_green_kubo_table_matches_reference(name, tmp_path):
    text = GK_CASES[name].replace("@DIR@", str(tmp_path))
    cfg = so.parse_script(text)
    nevery, nblock, fn, mode = _gk_line(text)
    o = so.Oracle(cfg)
    gk = so.GreenKubo(cfg, nevery, nblock, mode)
    u = DATA[f"{name}/u0"]
    nsteps = DATA[f"{name}/states"].shape[0]
    for _ in range(nsteps):
        u, flux = o.step_with_flux(u, None)   # psi's noise does not reach pi_xy here
        gk.observe(flux)
    lines = ["# nsample tau mode_index kx ky S_mean"]
    for ti in range(gk.ntau):
        tau = float((ti + 1) * nevery) * cfg.dt
        for mi, (nx, ny) in enumerate(gk.modes):
            kx = 2.0 * 3.14159265358979323846 * float(nx) / cfg.length[0]
            ky = 2.0 * 3.14159265358979323846 * float(ny) / cfg.length[1]
            lines.append(f"{gk.nsample} {tau:.16e} {mi} {kx:.16e} {ky:.16e} {gk.sums[ti, mi] / gk.nsample:.16e}")
    _compare_gk("\n".join(lines) + "\n", str(DATA[f"{name}/file/{fn}"]), 1e-10)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", sorted(GK_CASES))
def test_engine_green_kubo_file_matches_reference(name, precision, tmp_path):
    import shhd_b200 as sb
    from shhd_b200.measures import run_script_measures
    text = GK_CASES[name].replace("@DIR@", str(tmp_path))
    cfg = sb.config_from_script(text)
    cfg.precision = precision
    _nevery, _nblock, fn, _mode = _gk_line(text)
    with sb.Engine(cfg) as eng:
        eng.set_state(DATA[f"{name}/u0"])
        run_script_measures(eng, text)
    with open(tmp_path / fn) as f:
        _compare_gk(f.read(), str(DATA[f"{name}/file/{fn}"]), 1e-10 if precision == 0 else 1e-3)
