"""The whole-step entry points (fs_ctx_create / fs_step / fs_batch_run): the
outer loop driven from C++ gives the reference's states, the Python
stepper's states bit for bit, and the same results when several cases are
stepped at once."""
import numpy as np
import pytest

from test_gpu_step import _compare

pytestmark = pytest.mark.gpu

KEYS = ("rho", "u", "v", "w", "T_g", "Y_fuel", "Y_O2", "Y_H2O", "T_s", "k_turb", "eps_turb",
        "nu_t", "phi", "omega", "q_rad", "q_rad_gas", "T_soil", "S_pyro_b", "S_dry_b",
        "Q_gconv_b", "p_T_s", "p_m_solid", "p_m_water", "p_m_char")


def test_fs_step_matches_reference(ref_tiny):
    """Ten fs_step calls on the 32 x 8 x 12 case: every field within 1e-9 of
    the reference's run after the captured steps, the same dt sequence."""
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.ctx import StepContext
    s = StepContext(TINY, projection_cg_rtol=1e-13, proj_maxiter=400)
    try:
        dts = []
        for n in range(1, 11):
            out = s.step(1)
            assert out.steps == 1 and out.step_count == n and not out.finished
            dts.append(out.dt)
            if f"s{n}" in ref_tiny:
                _compare(s.state(), ref_tiny[f"s{n}"], f"fs_step {n}")
        assert np.allclose(dts, ref_tiny["trace"]["dt"], rtol=1e-12, atol=0.0)
    finally:
        s.close()


@pytest.mark.parametrize("form", ["plain", "mixed"])
def test_fs_step_equals_python_stepper(form):
    """Three steps through fs_step and through Tier3Solver.step (the same
    kernels in the same order): identical states, with and without the DOM
    on its own stream."""
    from firewebapp_b200.cases import SMOKE
    from firewebapp_b200.ctx import StepContext
    from firewebapp_b200.solver import Tier3Solver
    py = Tier3Solver(SMOKE, form=form)
    cs = [StepContext(SMOKE, form=form), StepContext(SMOKE, form=form, overlap_dom=False)]
    try:
        for _ in range(3):
            py.step()
        want = py.state()
        for c in cs:
            out = c.step(3)
            assert out.steps == 3 and abs(out.t - py.t) == 0.0
            got = c.state()
            for k in KEYS:
                assert np.array_equal(got[k], want[k]), (form, k)
            assert np.array_equal(got["p_prev"], want["p_prev"])
    finally:
        py.close()
        for c in cs:
            c.close()


def test_batch_run_equals_single_runs():
    """fs_batch_run steps three different cases at once (own host thread and
    streams each): every case ends where stepping it alone ends."""
    from firewebapp_b200.cases import SMOKE, TINY
    from firewebapp_b200.ctx import StepContext, batch_run
    cases = [(TINY, "plain"), (SMOKE, "plain"), (TINY, "mixed")]
    alone = []
    for case, form in cases:
        c = StepContext(case, form=form)
        c.step(3)
        alone.append(c.state())
        c.close()
    ctxs = [StepContext(case, form=form) for case, form in cases]
    try:
        outs = batch_run(ctxs, 3)
        assert [o.steps for o in outs] == [3, 3, 3]
        for c, want in zip(ctxs, alone):
            got = c.state()
            for k in KEYS:
                assert np.array_equal(got[k], want[k]), k
    finally:
        for c in ctxs:
            c.close()


def test_fs_ctx_write_then_step():
    """A field written through fs_ctx_write is the one the next step reads
    (the same change made to the Python stepper gives the same state)."""
    from firewebapp_b200.cases import SMOKE
    from firewebapp_b200.ctx import StepContext
    from firewebapp_b200.solver import Tier3Solver
    import torch
    py = Tier3Solver(SMOKE)
    c = StepContext(SMOKE)
    try:
        py.step()
        c.step(1)
        tg = c.read("T_g") * 1.01
        c.write("T_g", tg)
        py.f["T_g"].copy_(torch.as_tensor(tg))
        py.step()
        c.step(1)
        want, got = py.state(), c.state()
        for k in ("T_g", "rho", "u", "omega", "q_rad"):
            assert np.array_equal(got[k], want[k]), k
    finally:
        py.close()
        c.close()
