"""Failure detection mirrored as status codes, driven from host-side inputs
(no GPU fault): non-finite fields, a pressure solve that cannot converge in
its iteration budget, and the learned solve's forced fallback."""
import ctypes as C

import numpy as np
import pytest
import torch

from firewebapp_b200._lib import FireStepError

pytestmark = pytest.mark.gpu


def test_nan_gas_temperature_raises_like_the_reference():
    """spread_3d.py:1927-1932: NaN/Inf in T_g raises RuntimeError at the dt check."""
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.solver import Tier3Solver
    s = Tier3Solver(TINY)
    s.step()
    s.f["T_g"][3, 2, 5] = float("nan")
    with pytest.raises(RuntimeError, match="NaN/Inf"):
        s.step()
    s.close()


@pytest.mark.parametrize("fp32", [0, 1])
def test_dom_non_finite_input_returns_status_2(fp32):
    """NaN temperatures make G non-finite; the path-8 source iteration's
    device-side test reports it as FS_ENONFINITE, and the context stays usable."""
    from test_gpu_kernels import _dom_solves
    import test_gpu_kernels as K
    orig = K.dev
    calls = {"n": 0}

    def poisoned(a, dtype=torch.float64):
        t = orig(a, dtype)
        calls["n"] += 1
        if calls["n"] in (1, 2):  # T_s and T_g of the first solve, every 97th cell
            t.view(-1)[::97] = float("nan")
        return t

    K.dev = poisoned
    try:
        with pytest.raises(FireStepError) as ei:
            _dom_solves(8, fp32, 29, 40, 48, seed=5, calls=1)
    finally:
        K.dev = orig
    assert ei.value.status == 2
    # a clean solve on the same device afterwards works
    out = _dom_solves(8, fp32, 29, 40, 48, seed=5, calls=1)
    assert np.all(np.isfinite(out[0][0]))


def test_projection_iteration_cap_returns_status_3():
    """projection_3d.py:785-790 raises on BiCGSTAB failure; here a solve that
    cannot meet its tolerance within maxiter returns FS_ENOCONV (3)."""
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.solver import Tier3Solver
    s = Tier3Solver(TINY)
    for _ in range(3):
        s.step()
    s.rtol, s.proj_maxiter = 1e-14, 1
    with pytest.raises(FireStepError) as ei:
        s.step()
    assert ei.value.status == 3
    s.close()


def test_learned_stall_falls_back_and_converges():
    """A network switched off (output scale 0) with a strict stall test falls
    back to the V-cycle within the solve and still reaches the tolerance."""
    from firewebapp_b200.cases import TINY
    from firewebapp_b200.learned import fcg_stats, init_params
    from firewebapp_b200.solver import Tier3Solver
    s = Tier3Solver(TINY, form="learned", learned_weights=init_params(2), learned_stall=0.5,
                    learned_max=50)
    s.net.set_output_scale(0.0)
    fell = 0
    for _ in range(5):
        assert s.step()
        st = fcg_stats(s)
        fell += int(st["fell_back"])
        if st["fell_back"]:
            assert st["learned_iters"] >= 3 and st["vcycle_iters"] >= 1
    assert fell >= 1 and fcg_stats(s)["fallbacks_total"] == fell
    s.close()


@pytest.mark.parametrize("kernel", [1, 2])
@pytest.mark.parametrize("fp32", [0, 1])
def test_dom_hand_off_wait_runs_out_with_status_4(fp32, kernel):
    """Path 8's CTAs wait for one another's rows with bounded waits.  With the
    test switch one CTA withholds a row (a fill that nothing else sends), the
    next CTA's wait runs out, the solve returns FS_ETIMEOUT (4) instead of
    hanging, and the same object then solves normally; with either sweep
    kernel (pencil per thread on 29 levels in CTAs of 3 rows, lane column on
    40 levels in CTAs of 4)."""
    from gpu_helpers import Grid, call, dev, host, lib, stream
    from firewebapp_b200._lib import dbl_array, ptr
    from firewebapp_b200.quadrature import level_symmetric
    om, wq = level_symmetric(8)
    nz, ny, nx = (29, 40, 48) if kernel == 1 else (40, 40, 48)
    rng = np.random.default_rng(3)
    g = Grid(nz, ny, nx, 0.5, 0.5, np.full(nz, 0.1))
    h = C.c_void_p()
    call("fs_dom_create", g.ref, om.shape[0], dbl_array(om[:, 0]), dbl_array(om[:, 1]),
         dbl_array(om[:, 2]), dbl_array(wq), 0.5, C.byref(h))
    shape = (nz, ny, nx)
    Ts = dev(300.0 + 900.0 * rng.random(shape) ** 4)
    Tg = dev(300.0 + 1500.0 * rng.random(shape) ** 6)
    a = dev(np.where(rng.random(shape) < 0.3, 0.002 * rng.random(shape), 0.0))
    zero = dev(np.zeros(shape))
    M = dev(0.05 + 0.1 * rng.random(shape))
    rho = dev(np.ones(shape))
    Tsoil = dev(np.full((ny, nx), 300.0))
    qs, qg = torch.zeros_like(Ts), torch.zeros_like(Ts)
    qsoil = torch.zeros((ny, nx), dtype=torch.float64, device="cuda")

    def solve():
        return lib().fs_dom_solve(h, ptr(Ts), ptr(Tg), ptr(a), ptr(zero), 5000.0, 300.0,
                                  ptr(Tsoil), ptr(zero), ptr(rho), ptr(M), ptr(qs), ptr(qg),
                                  ptr(qsoil), stream())
    try:
        if fp32:
            call("fs_dom_set_precision", h, 1)
        call("fs_dom_set_sweep_mode", h, 8, 0)
        call("fs_dom_set_sweep_kernel", h, kernel)
        assert solve() == 0
        assert lib().fs_dom_sweep_kernel(h) == kernel
        call("fs_dom_set_wait_test", h, 5)
        assert solve() == 4
        assert b"gave up" in lib().fs_last_error()
        call("fs_dom_set_wait_test", h, -1)
        assert solve() == 0
        assert np.all(np.isfinite(host(qs))) and np.all(np.isfinite(host(qg)))
    finally:
        lib().fs_dom_destroy(h)
