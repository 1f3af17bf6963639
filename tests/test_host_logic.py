"""Host-side logic that needs no GPU: initial conditions restated from the
reference's drivers, checked against the reference's own output."""
import numpy as np

from conftest import load_golden


def test_ink_particle_positions_match_reference():
    from edgeb200.sim import ink_particles
    d = load_golden("lp_init_positions")
    for case in (0, 1):
        pos = ink_particles(case, 300).astype(np.float32)
        np.testing.assert_array_equal(pos, d[f"pos_case{case}"])


def test_driver_cases_cover_the_reference():
    """run_edge.py has cases 0-4; the other drivers cases 0-1."""
    from edgeb200.driver import CASES
    edge = sorted(c for c, v in CASES.items() if v.get("only", "edge") == "edge")
    ge = sorted(c for c, v in CASES.items() if v.get("only", "ge") == "ge")
    assert edge == [0, 1, 2, 3, 4]
    assert ge == [0, 1]
    assert CASES[4]["res"] == (256, 512, 256) and CASES[4]["lp"]["num"] == 4000000
