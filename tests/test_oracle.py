"""The oracle against the reference's own outputs (CPU).

The golden fixtures come from the reference's unmodified sources
(tests/golden/make_golden.py); the numpy restatement must reproduce the RHS
and two integrator steps of every case, with the reference's own noise
replayed, to FP64 round-off.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import load_golden

CASES = load_golden()
TOL = 1e-13


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_rhs_matches_reference(name):
    c = CASES[name]
    cfg = so.parse_script(c["script"])
    det = so.Oracle(cfg).rhs(c["u0"])
    assert so.rel_l2(det, c["det"]) < TOL


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_steps_match_reference(name):
    c = CASES[name]
    cfg = so.parse_script(c["script"])
    o = so.Oracle(cfg)
    u = c["u0"]
    for s in range(c["states"].shape[0]):
        u = o.step(u, (c["noise"][s, 0], c["noise"][s, 1]))
        assert so.rel_l2(u, c["states"][s]) < TOL, f"step {s}"


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_noise_has_the_restated_structure(name):
    """psi noise is sigma(k) * xi with conjugate pairs on kx = 0; j noise is -i k . pi.

    Rebuild xi from the reference's psi draws and check that the restated
    mapping returns the same field; for momentum check div-free structure of
    the stress form (the RHS is a k-linear map of a symmetric stress).
    """
    c = CASES[name]
    cfg = so.parse_script(c["script"])
    o = so.Oracle(cfg)
    g = o.geo
    n = cfg.num_order_parameters
    sa = c["noise"][0, 0]
    if cfg.noise_order_parameter and n > 0:
        pref = 2.0 * cfg.kBT * cfg.chi * g.grid_size ** 2 / g.volume
        xis = []
        for a in range(n):
            sig = np.sqrt(0.5 * pref * cfg.mobility[a] * g.k2)
            with np.errstate(divide="ignore", invalid="ignore"):
                xis.append(np.where(sig > 0, sa[1 + a] / np.where(sig > 0, sig, 1.0), 0.0))
        rebuilt = o.noise_from_normals(xis, [np.zeros_like(sa[0])] * 3)
        for a in range(n):
            assert so.rel_l2(rebuilt[1 + a], sa[1 + a]) < 1e-14
    # noise vanishes outside the active set and at k = 0
    assert np.all(sa[:, ~g.active] == 0)
    assert np.all(sa[:, 0, 0] == 0)


def test_philox_normals_statistics():
    ids = np.arange(200000, dtype=np.uint64)
    za, zb = so.philox_normals(1234, 0, 7, so.psi_stream(0), ids)
    for z in (za, zb):
        assert abs(z.real.mean()) < 0.01 and abs(z.imag.mean()) < 0.01
        assert abs(z.real.var() - 1) < 0.01 and abs(z.imag.var() - 1) < 0.01
        assert abs(np.mean(z.real * z.imag)) < 0.01
    assert abs(np.mean(za.real * zb.real)) < 0.01
    # different streams, steps, members and seeds are different realisations
    for other in (so.philox_normals(1234, 0, 7, so.psi_stream(1), ids)[0], so.philox_normals(1234, 0, 8, so.psi_stream(0), ids)[0],
                  so.philox_normals(1234, 1, 7, so.psi_stream(0), ids)[0], so.philox_normals(99, 0, 7, so.psi_stream(0), ids)[0]):
        assert abs(np.mean(za.real * other.real)) < 0.01


def test_philox4x32_known_answer():
    """Philox4x32-10 known-answer vectors published with Random123 (kat_vectors)."""
    out = so.philox4x32_10(0, 0, 0, 0, 0, 0)
    assert [int(v) for v in out] == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    m = 0xFFFFFFFF
    out = so.philox4x32_10(m, m, m, m, m, m)
    assert [int(v) for v in out] == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    out = so.philox4x32_10(0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344, 0xA4093822, 0x299F31D0)
    assert [int(v) for v in out] == [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_symmetry_projection_is_idempotent():
    c = CASES["srk3_compressible_n2"]
    cfg = so.parse_script(c["script"])
    o = so.Oracle(cfg)
    u = c["states"][0]
    assert np.array_equal(o.enforce_real_symmetry(u), u)
