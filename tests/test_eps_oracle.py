"""Extended-period oracle: pinned to the reference's EPANET-replica EpsDriver
(fixture tests/golden/eps_ref.npz, made by `make_golden.py eps`), and its
adjoint through time checked against central differences."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.eps import EpsOracle  # noqa: E402


@pytest.fixture(scope="module")
def case():
    net, inp, ref = load("eps_ref")
    return net, inp, ref


def _rh(net, B):
    return np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), (B, net.N)).copy()


def test_eps_oracle_matches_reference_eps_driver(case):
    """Tank levels, junction heads and flows of every hourly frame agree with
    dgga.eps.EpsDriver (which polishes nothing and stops at accuracy 1e-5;
    the oracle's polished steps sit at the same fixed points)."""
    net, inp, ref = case
    T = int(inp["T"])
    eo = EpsOracle(net)
    run = eo.run(inp["demand"], _rh(net, 1), np.asarray(net.tank_h0)[None], accuracy=1e-9)
    assert ref["t_sec"].tolist() == [3600 * t for t in range(T)]
    tn = np.asarray(net.tank_node)
    junc = np.asarray(net.node_type) == 0
    assert np.abs(ref["head_ft"][:, tn] - run["tank_head"][:T, 0]).max() < 1e-7
    assert np.abs(ref["head_ft"][:, junc] - run["head"][:, 0][:, junc]).max() < 1e-7
    assert np.abs(ref["flow_int_cfs"] - run["flow"][:, 0]).max() < 1e-7
    # the tanks do move (the pin is not vacuous)
    assert np.abs(run["tank_head"][-1] - run["tank_head"][0]).max() > 0.05


def test_eps_oracle_adjoint_matches_central_difference(case):
    net, inp, _ = case
    T, B = 3, 2
    eo = EpsOracle(net)
    rng = np.random.default_rng(4)
    dem = inp["demand"][:T, :1].repeat(B, 1) * rng.uniform(0.9, 1.1, (T, B, net.N))
    rh = _rh(net, B)
    th0 = np.broadcast_to(np.asarray(net.tank_h0), (B, len(net.tank_node))).copy()
    r = np.broadcast_to(np.asarray(net.r_hw), (B, net.L)).copy()
    sens = np.flatnonzero(np.asarray(net.node_type) == 0)[::7]
    tn = np.asarray(net.tank_node)
    wq = rng.normal(size=net.L)

    def loss_parts(run):
        return ((run["head"][:, :, sens] ** 2).sum() + (run["tank_head"][-1] ** 2).sum()
                + (run["flow"] * wq).sum())

    def loss(d=dem, h0=th0, rr=r):
        return loss_parts(eo.run(d, rh, h0, r=rr, accuracy=1e-12))

    run = eo.run(dem, rh, th0, r=r, accuracy=1e-12)
    gH = np.zeros((T, B, net.N))
    gH[:, :, sens] = 2.0 * run["head"][:, :, sens]
    gQ = np.broadcast_to(wq, (T, B, net.L)).copy()
    gE = np.zeros((T, B, net.N))
    gT = np.zeros((T + 1, B, tn.size))
    gT[T] = 2.0 * run["tank_head"][T]
    g_dem, g_rh, g_h0, g_ke, g_r = eo.backward(run, gH, gQ, gE, gT)
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
