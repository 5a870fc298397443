"""Pump-parameter gradient pin: the oracle's pump theta (speed, curve H0,
curve R) against the reference's CPU implicit adjoint with pump theta
(ImplicitGGASolve, dgga/autodiff.py:609-756; fixture tests/golden/pump_ref.npz,
`make_golden.py pumps`) on a network with power-function, custom-curve,
no-curve and constant-horsepower pumps, plus a finite-difference check of the
d hloss / d theta formulas through the oracle's own forward."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.gga import Model  # noqa: E402


def pump_loss_grads(m, net, inp, accuracy=1e-7):
    """Forward + polish at the model's pump parameters and the adjoint of
    L = sum h[sensors]^2 + sum h[pump n2]^2 + sum q[pumps]^2."""
    d, rh = inp["demand"], inp["res_head"]
    out, st = m.implicit(d, rh, ke=inp["ke"], accuracy=accuracy)
    B = d.shape[0]
    pl = np.asarray(net.pump_link)
    pn2 = np.asarray(net.link_n2)[pl]
    H, q = out["head_ft"], out["flow_cfs"]
    gH = np.zeros((B, net.N))
    for idx in (np.asarray(inp["sensors"]), pn2):     # repeated nodes accumulate
        for b in range(B):
            np.add.at(gH[b], idx, 2.0 * H[b, idx])
    gQ = np.zeros((B, net.L))
    gQ[:, pl] = 2.0 * q[:, pl]
    loss = (H[:, inp["sensors"]] ** 2).sum(1) + (H[:, pn2] ** 2).sum(1) + (q[:, pl] ** 2).sum(1)
    g = m.backward(st, gH, gQ, np.zeros((B, net.N)), pumps=True)
    return out, loss, g


def test_oracle_pump_theta_matches_reference():
    net, inp, ref = load("pump_ref")
    m = Model(net).with_pumps(inp["speed"], inp["pump_h0"], inp["pump_r"])
    out, _, g = pump_loss_grads(m, net, inp)
    assert (out["status"] == inp["status"]).all()
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-9
    for gi, key in ((g[0], "g_demand"), (g[1], "g_res_head"), (g[3], "g_rhw"), (g[4], "g_speed"),
                    (g[5], "g_h0"), (g[6], "g_r")):
        R = ref[key]
        assert np.abs(gi - R).max() <= 1e-9 * np.abs(R).max(), (key, np.abs(gi - R).max())
    pl = np.asarray(net.pump_link)
    # every curve kind with a theta derivative is exercised (no-curve has none)
    assert (np.abs(ref["g_speed"][:, pl[[0, 1, 3]]]) > 1e3).all()


def test_oracle_pump_theta_finite_difference():
    """Central differences of the loss in each pump parameter of scenario 0."""
    net, inp, ref = load("pump_ref")
    sp, h0, rp = inp["speed"].copy(), inp["pump_h0"].copy(), inp["pump_r"].copy()
    one = {k: v[:1] for k, v in inp.items() if k in ("demand", "res_head")}
    one.update(ke=inp["ke"], sensors=inp["sensors"])
    m = Model(net).with_pumps(sp, h0, rp)
    _, _, g = pump_loss_grads(m, net, one)
    pl = np.asarray(net.pump_link)
    checks = [(0, pl[0]), (0, pl[1]), (0, pl[3]), (1, pl[0]), (2, pl[0]), (2, pl[3])]
    for which, k in checks:
        base = [sp, h0, rp][which]
        eps = 1e-6 * max(abs(base[k]), 1.0)
        vals = []
        for sgn in (1.0, -1.0):
            th = [sp.copy(), h0.copy(), rp.copy()]
            th[which][k] += sgn * eps
            _, loss, _ = pump_loss_grads(Model(net).with_pumps(*th), net, one)
            vals.append(loss[0])
        fd = (vals[0] - vals[1]) / (2.0 * eps)
        an = g[4 + which][0, k]
        assert abs(fd - an) <= 1e-5 * max(abs(an), 1.0), (which, k, fd, an)


def test_oracle_chp_clamp_matches_reference():
    """A constant-HP pump feeding a dead end of tiny demand sits on its CBIG
    clamp branch; the exact Jacobian there (-CBIG where the GGA matrix has
    +CBIG, dgga/autodiff.py:186-193) gives the reference's CPU-adjoint
    gradients (fixture tests/golden/chp_ref.npz), and the assembled one does
    not."""
    net, inp, ref = load("chp_ref")
    m = Model(net).with_pumps(inp["speed"], inp["pump_h0"], inp["pump_r"])
    out, _, g = pump_loss_grads(m, net, inp)
    assert (out["status"] == inp["status"]).all()
    pl = np.asarray(net.pump_link)
    assert m.chp_clamp(out["flow_cfs"], out["status"])[:, pl[3]].all()
    for gi, key in ((g[0], "g_demand"), (g[1], "g_res_head"), (g[3], "g_rhw"), (g[4], "g_speed"),
                    (g[5], "g_h0"), (g[6], "g_r")):
        R = ref[key]
        assert np.abs(gi - R).max() <= 1e-9 * np.abs(R).max(), (key, np.abs(gi - R).max())
    m.chp_clamp = lambda q, S: np.zeros(q.shape, dtype=bool)      # the assembled Jacobian
    _, _, g = pump_loss_grads(m, net, inp)
    assert np.abs(g[0] - ref["g_demand"]).max() > 0.5 * np.abs(ref["g_demand"]).max()
