"""Checkpoint/resume: a run restored from a checkpoint continues bit-identically
(the reference has no checkpoint; this pins the build's own format)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_checkpoint_resume_is_bit_identical(tmp_path):
    from firewebapp_b200.api import load_checkpoint, save_checkpoint
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.solver import Tier3Solver
    a = Tier3Solver(TINY, projection_cg_rtol=1e-10)
    for _ in range(3):
        a.step()
    ck = save_checkpoint(a, tmp_path / "ck.npz")
    for _ in range(2):
        a.step()
    want = a.state()
    b = load_checkpoint(ck)
    assert b.step_count == 3
    for _ in range(2):
        b.step()
    got = b.state()
    for k, v in want.items():
        assert np.array_equal(np.asarray(got[k]), np.asarray(v)), k
    assert b.t == a.t and b.front_x == a.front_x
    a.close()
    b.close()
