"""Host initial-condition styles reproduce the reference's own initial states (CPU)."""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import load_golden

CASES = load_golden()
SUPPORTED = ("uniform", "equilibrium/gaussian", "equilibrium/gaussian/compressible")


def _supported(script):
    for line in script.splitlines():
        t = line.split()
        if t and t[0] == "set":
            style = t[2] if t[1] in ("density", "rho") else t[3]
            if style not in SUPPORTED:
                return False
    return True


@pytest.mark.parametrize("name", sorted(n for n, c in CASES.items() if _supported(c["script"])))
def test_initial_state_matches_reference(name):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state
    c = CASES[name]
    cfg = sb.config_from_script(c["script"])
    u = initial_state(cfg, c["script"])
    assert u.shape == c["u0"].shape
    assert so.rel_l2(u, c["u0"]) < 1e-15
