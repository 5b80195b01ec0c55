"""Host initial-condition styles reproduce the reference's own initial states and errors (CPU).

Two fixture sets, both produced by the reference's own code (tests/golden/make_golden.py):
the step cases' initial states, and initial-condition-only cases that reach every
built-in style, the default seeds, last-command-wins and the reference's refusals.
"""
import numpy as np
import pytest

import shhd_oracle as so
from helpers import load_golden, load_initial_golden

CASES = load_golden()
IC_CASES = load_initial_golden()


@pytest.mark.parametrize("name", sorted(CASES))
def test_initial_state_matches_reference(name):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state
    c = CASES[name]
    cfg = sb.config_from_script(c["script"])
    u = initial_state(cfg, c["script"])
    assert u.shape == c["u0"].shape
    assert so.rel_l2(u, c["u0"]) < 1e-15


@pytest.mark.parametrize("name", sorted(IC_CASES))
def test_initial_styles_match_reference(name):
    import shhd_b200 as sb
    from shhd_b200.initial import initial_state
    c = IC_CASES[name]
    cfg = sb.config_from_script(c["script"])
    if c["error"] is not None:
        with pytest.raises(ValueError) as ei:
            initial_state(cfg, c["script"])
        assert str(ei.value) == c["error"]
    else:
        u = initial_state(cfg, c["script"])
        assert u.shape == c["u0"].shape
        assert so.rel_l2(u, c["u0"]) < 1e-15
