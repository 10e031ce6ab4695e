"""CPU checks of the learned preconditioner's oracle and parameter layout."""
import numpy as np

from oracle import unet as U


def test_parameter_layout_agrees():
    from firewebapp_b200 import learned, _lib
    assert learned.n_params() == U.n_params() == 587953
    assert int(_lib.lib().fs_unet_nparams()) == U.n_params()
    lay, hw, hb, n = U.param_layout()
    assert [(c, o) for _nm, c, o, _w, _b in lay] == list(learned.CONV_LAYERS)
    assert hb == n - 1 and hw == n - 17


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = U.init_params(3)
    lay, hw, hb, _n = U.param_layout()
    for _name, _cin, cout, _w, b in lay:
        p[b:b + cout] = rng.uniform(-0.1, 0.1, cout)
    r = rng.standard_normal((5, 6, 7))
    tau = rng.standard_normal((5, 6, 7))
    _L, g, _z = U.loss_and_grad(p, r, tau, rnd=False)
    idx = [hw + 3, hb]
    for _name, cin, cout, w, b in lay:
        idx += [w + 13 * cin * cout + 5, w + 4 * cin * cout + 1, b + 1]
    checked = 0
    for i in idx:
        h = 1e-6
        pp = p.copy(); pp[i] += h
        pm = p.copy(); pm[i] -= h
        fd = (U.loss_and_grad(pp, r, tau, rnd=False)[0]
              - U.loss_and_grad(pm, r, tau, rnd=False)[0]) / (2 * h)
        assert abs(g[i] - fd) <= 1e-6 * max(abs(fd), 1e-3), (i, g[i], fd)
        checked += g[i] != 0.0
    assert checked >= 15


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1e-3, 0.0])
    y = U.bf16(x)
    assert y[0] == 1.0 and y[1] == 1.0            # tie to even
    assert y[2] == 1.0 + 2 ** -6                  # tie to even (up)
    assert y[3] == -2.5 and y[5] == 0.0
    assert abs(y[4] - 1e-3) <= 2 ** -9 * 1e-3


def test_packaged_weights_have_the_layout():
    from firewebapp_b200 import learned
    d = np.load(learned.WEIGHTS)
    assert d["params"].dtype == np.float32 and d["params"].size == learned.n_params()
    assert np.all(np.isfinite(d["params"])) and float(d["target_scale"]) > 0.0
