"""Unrolled-K pin: the oracle's K fixed GGA iterations and its explicit
reverse pass against the reference's solve_unrolled and its autograd
gradients (fixture tests/golden/unrolled_ref.npz, `make_golden.py
unrolled`) and with a warm start and frozen statuses (unrolled_warm_ref.npz,
`make_golden.py unrolled_warm`), plus central differences of the oracle's
own K-iteration map."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.gga import Model  # noqa: E402
from oracle.unrolled import Unrolled  # noqa: E402


def unrolled_loss_adjoints(net, inp, out):
    """Output adjoints of L = sum h[sensors]^2 + sum q[pumps]^2 + sum e[emitters]^2."""
    B = out["head_ft"].shape[0]
    sens = np.asarray(inp["sensors"])
    pl = np.asarray(net.pump_link)
    emn = np.flatnonzero(np.asarray(net.node_ke) > 0)
    gH, gQ, gE = np.zeros((B, net.N)), np.zeros((B, net.L)), np.zeros((B, net.N))
    for b in range(B):
        np.add.at(gH[b], sens, 2.0 * out["head_ft"][b, sens])
    gQ[:, pl] = 2.0 * out["flow_cfs"][:, pl]
    gE[:, emn] = 2.0 * out["emitter_cfs"][:, emn]
    loss = ((out["head_ft"][:, sens] ** 2).sum(1) + (out["flow_cfs"][:, pl] ** 2).sum(1)
            + (out["emitter_cfs"][:, emn] ** 2).sum(1))
    return gH, gQ, gE, loss


def test_oracle_unrolled_matches_reference():
    net, inp, ref = load("unrolled_ref")
    u = Unrolled(Model(net))
    out, st = u.forward(inp["demand"], inp["res_head"], ke=inp["ke"], K=int(inp["K"]))
    # unconverged K-iteration state: the two linear solvers' rounding, as raw GGA states
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-4
    assert np.abs(out["flow_cfs"] - ref["flow"]).max() < 1e-6
    gd, grh, gke, gr = u.backward(st, *unrolled_loss_adjoints(net, inp, out)[:3])
    junc = np.asarray(net.node_type) == 0
    for g, key, cols in ((gd, "g_demand", junc), (grh, "g_res_head", ~junc), (gke, "g_ke", junc)):
        R = ref[key][:, cols]
        assert np.abs(g[:, cols] - R).max() <= 1e-6 * np.abs(R).max(), key
    R = ref["g_rhw"]                                  # r_hw is [L]: the batch sum
    assert np.abs(gr.sum(0) - R).max() <= 1e-6 * np.abs(R).max()


def test_oracle_unrolled_central_difference():
    net, inp, _ = load("unrolled_ref")
    u = Unrolled(Model(net))
    d, rh = inp["demand"][:1], inp["res_head"][:1]
    K = int(inp["K"])
    out, st = u.forward(d, rh, K=K)
    gd, grh, _, gr = u.backward(st, *unrolled_loss_adjoints(net, inp, out)[:3])

    def loss(dd, rr=None):
        o, _ = u.forward(dd, rh, r=rr, K=K)
        return unrolled_loss_adjoints(net, inp, o)[3][0]

    # the K-iteration map is smooth only down to its rounding (about 1e-7 of
    # the loss after 8 unconverged iterations on a matrix with a 1e8 penalty),
    # so the steps are large: 1e-3 cfs of demand, 1e-3 of a resistance
    junc = np.flatnonzero(np.asarray(net.node_type) == 0)
    for p in junc[[3, 17, 40]]:
        eps = 1e-3
        dp, dm = d.copy(), d.copy()
        dp[0, p] += eps
        dm[0, p] -= eps
        fd = (loss(dp) - loss(dm)) / (2 * eps)
        assert abs(fd - gd[0, p]) <= 2e-3 * abs(gd[0, p]), (p, fd, gd[0, p])
    r0 = np.asarray(net.r_hw, dtype=np.float64)
    for k in np.argsort(-np.abs(gr[0]))[:2]:
        eps = 1e-3 * r0[k]
        rp, rm = r0.copy(), r0.copy()
        rp[k] += eps
        rm[k] -= eps
        fd = (loss(d, rp) - loss(d, rm)) / (2 * eps)
        assert abs(fd - gr[0, k]) <= 2e-3 * abs(gr[0, k]), (k, fd, gr[0, k])


def test_oracle_unrolled_warm_matches_reference():
    """Warm start q0 / e0 (the reference's own converged flows at 90 %
    demand) and its final statuses frozen, K = 6."""
    net, inp, ref = load("unrolled_warm_ref")
    u = Unrolled(Model(net))
    S = np.asarray(inp["status"], dtype=np.int8)
    out, st = u.forward(inp["demand"], inp["res_head"], ke=inp["ke"], K=int(inp["K"]), S=S,
                        q0=inp["q0"], e0=inp["e0"])
    # the iterates of either code move by up to 1e-4 ft per iteration at the
    # fixed point (the 1e8 penalty of the closed links amplifies the linear
    # solves' rounding), so the state bars are those of the cold start
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-4
    assert np.abs(out["flow_cfs"] - ref["flow"]).max() < 1e-6
    assert np.abs(out["emitter_cfs"] - ref["emitter"]).max() < 1e-6
    gd, grh, gke, gr = u.backward(st, *unrolled_loss_adjoints(net, inp, out)[:3])
    junc = np.asarray(net.node_type) == 0
    for g, key, cols in ((gd, "g_demand", junc), (grh, "g_res_head", ~junc), (gke, "g_ke", junc)):
        R = ref[key][:, cols]
        assert np.abs(g[:, cols] - R).max() <= 1e-6 * np.abs(R).max(), key
    R = ref["g_rhw"]
    assert np.abs(gr.sum(0) - R).max() <= 1e-6 * np.abs(R).max()
