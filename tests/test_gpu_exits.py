"""The loop's exit tests (spread_3d.py:3413-3437) against the reference's own
runs (tests/golden/ref_exits.npz, tests/golden/make_exits.py): with no
ignition the flame body stays empty and the loop leaves after more than 50
such steps past the ignition window plus the 2 s bootstrap; with the bed
ending one cell after the ignition strip the front is at the bed's end and
the loop leaves in its first step.  Both steppers leave in the reference's
step (Tier3Solver.step returns False there; fs_step reports finished)."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_exits.npz"


@pytest.mark.parametrize("name", ["extinct", "front"])
def test_python_stepper_leaves_where_the_reference_does(name):
    from firewebapp_b200.cases import EXIT_CASES
    from firewebapp_b200.solver import Tier3Solver
    ref = np.load(GOLDEN)
    s = Tier3Solver(EXIT_CASES[name])
    try:
        for _ in range(400):
            if not s.step():
                break
        assert s.finished == "exit"
        assert s.step_count == int(ref[f"{name}/steps"])
        assert abs(s.t - float(ref[f"{name}/t"])) <= 1e-9 * max(1.0, float(ref[f"{name}/t"]))
    finally:
        s.close()


@pytest.mark.parametrize("name", ["extinct", "front"])
def test_fs_step_leaves_where_the_reference_does(name):
    from firewebapp_b200.cases import EXIT_CASES
    from firewebapp_b200.ctx import StepContext
    ref = np.load(GOLDEN)
    c = StepContext(EXIT_CASES[name])
    try:
        out = c.step(400)
        assert out.finished == 1
        assert out.steps == int(ref[f"{name}/steps"]) == out.step_count
        again = c.step(5)  # a finished loop takes no further steps
        assert again.steps == 0 and again.finished == 1
    finally:
        c.close()
