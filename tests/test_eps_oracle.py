"""Extended-period oracle: pinned to the reference's EPANET-replica EpsDriver
(fixtures tests/golden/eps_ref.npz and eps_events_ref.npz, made by
`make_golden.py eps` / `eps_events`), and its adjoint through time checked
against central differences."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.eps import EpsOracle  # noqa: E402


def _rh(net, B):
    return np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), (B, net.N)).copy()


@pytest.mark.parametrize("tag", ["eps_ref", "eps_events_ref"])
def test_eps_oracle_matches_reference_eps_driver(tag):
    """Frame times, tank levels, junction heads, flows and link statuses of
    every frame agree with dgga.eps.EpsDriver (which polishes nothing and
    stops at accuracy 1e-5; the oracle's polished frames sit at the same
    fixed points).  In eps_events the tanks fill: EpsDriver shortens steps
    at the fill times, tank links close and reopen, and a pump reopens from
    XHEAD, all carried from frame to frame."""
    net, inp, ref = load(tag)
    eo = EpsOracle(net)
    runs = eo.run(inp["demand"], _rh(net, 1), np.asarray(net.tank_h0)[None], accuracy=1e-9)
    fr = runs[0]
    assert fr["t"] == ref["t_sec"].tolist()
    tn = np.asarray(net.tank_node)
    junc = np.asarray(net.node_type) == 0
    head = np.stack(fr["head"])
    assert np.abs(ref["head_ft"][:, tn] - np.stack(fr["tank_head"])).max() < 1e-7
    assert np.abs(ref["head_ft"][:, junc] - head[:, junc]).max() < 1e-7
    assert np.abs(ref["flow_int_cfs"] - np.stack(fr["flow"])).max() < 1e-7
    np.testing.assert_array_equal(ref["status"], (np.stack(fr["status"]) > 2).astype(np.int8))
    th = np.stack(fr["tank_head"])
    assert np.abs(th[-1] - th[0]).max() > 0.05          # the tanks do move
    if tag == "eps_events_ref":
        assert any(t % 3600 for t in fr["t"])            # shortened steps
        assert (np.diff(ref["status"], axis=0) != 0).any()  # statuses change


def test_eps_oracle_adjoint_matches_central_difference():
    net, inp, _ = load("eps_ref")
    P, B = 3, 2
    eo = EpsOracle(net)
    rng = np.random.default_rng(4)
    dem = inp["demand"][:P, :1].repeat(B, 1) * rng.uniform(0.9, 1.1, (P, B, net.N))
    rh = _rh(net, B)
    th0 = np.broadcast_to(np.asarray(net.tank_h0), (B, len(net.tank_node))).copy()
    r = np.broadcast_to(np.asarray(net.r_hw), (B, net.L)).copy()
    sens = np.flatnonzero(np.asarray(net.node_type) == 0)[::7]
    wq = rng.normal(size=net.L)

    def grads(runs):
        gH = [[np.where(np.isin(np.arange(net.N), sens), 2.0 * h, 0.0) for h in fr["head"]]
              for fr in runs]
        gQ = [[wq for _ in fr["flow"]] for fr in runs]
        gE = [[np.zeros(net.N) for _ in fr["flow"]] for fr in runs]
        gT = [[np.zeros(len(net.tank_node)) for _ in fr["flow"]] for fr in runs]
        for fr, g in zip(runs, gT):
            g[-1] = 2.0 * fr["tank_head"][-1]
        return gH, gQ, gE, gT

    def loss_of(runs):
        tot = 0.0
        for fr in runs:
            for h, q in zip(fr["head"], fr["flow"]):
                tot += (h[sens] ** 2).sum() + (q * wq).sum()
            tot += (fr["tank_head"][-1] ** 2).sum()
        return tot

    def loss(d=dem, h0=th0, rr=r):
        return loss_of(eo.run(d, rh, h0, r=rr, accuracy=1e-12))

    runs = eo.run(dem, rh, th0, r=r, accuracy=1e-12)
    g_dem, g_rh, g_h0, g_ke, g_r = eo.backward(runs, *grads(runs), P=P)
    checks = []
    j = int(sens[1])
    for (t, b) in ((0, 0), (2, 1)):
        eps = 1e-3 * dem[t, b, j]
        dp, dm = dem.copy(), dem.copy()
        dp[t, b, j] += eps
        dm[t, b, j] -= eps
        checks.append((g_dem[t, b, j], (loss(d=dp) - loss(d=dm)) / (2 * eps)))
    for b, i in ((0, 0), (1, 2)):
        eps = 1e-5  # the tank pathway is strongly curved: small step
        hp, hm = th0.copy(), th0.copy()
        hp[b, i] += eps
        hm[b, i] -= eps
        checks.append((g_h0[b, i], (loss(h0=hp) - loss(h0=hm)) / (2 * eps)))
    k = int(np.argmax(np.asarray(net.r_hw)))
    eps = 1e-4 * r[0, k]
    rp, rm = r.copy(), r.copy()
    rp[0, k] += eps
    rm[0, k] -= eps
    checks.append((g_r[0, k], (loss(rr=rp) - loss(rr=rm)) / (2 * eps)))
    for an, fd in checks:
        assert abs(an - fd) <= 1e-5 * max(abs(fd), 1e-3), (an, fd)
