"""Extended-period run on the GPU (wdsgpu_b200.eps.eps_solve) against the
reference's EpsDriver (fixture tests/golden/eps_events_ref.npz: small tanks
that fill, shortened steps, tank links and a pump changing status) and the
oracle composition (oracle/eps.py, itself pinned to EpsDriver): frame times,
trajectory and statuses, adjoint through time, and central differences."""
import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.eps import EpsOracle  # noqa: E402

pytestmark = pytest.mark.gpu

HEAD_ATOL_FT = 1e-9 / 0.3048      # 1e-9 m
GRAD_RTOL = 1e-6


def _frames(out, b):
    v = out["valid"][:, b].cpu().numpy()
    f = lambda k: out[k][:, b].detach().cpu().numpy()[v]
    return dict(t=out["t_sec"][:, b].cpu().numpy()[v].tolist(), head=f("head"), flow=f("flow"),
                tank_head=f("tank_head"), status=f("status"))


@pytest.fixture(scope="module")
def setup(cuda):
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("eps_ref")
    P, B = 4, 3
    rng = np.random.default_rng(8)
    dem = inp["demand"][:P, :1].repeat(B, 1) * rng.uniform(0.85, 1.15, (P, B, net.N))
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), (B, net.N)).copy()
    th0 = np.broadcast_to(np.asarray(net.tank_h0), (B, len(net.tank_node))).copy()
    th0 = th0 + rng.uniform(-0.5, 0.5, th0.shape)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    return net, s, dem, rh, th0


def test_eps_events_match_reference_eps_driver(cuda):
    """Every frame of EpsDriver on the small-tank network: the same frame
    times (steps shortened where a tank fills), the same link statuses, and
    heads and flows at the reference's unpolished accuracy; against the
    oracle's polished frames within 1e-9 m."""
    from wdsgpu_b200.eps import eps_solve
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load("eps_events_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    rh = np.nan_to_num(net.fixed_head_ft_at(0))[None]
    out = eps_solve(s, inp["demand"], rh, accuracy=1e-9)
    fr = _frames(out, 0)
    assert fr["t"] == ref["t_sec"].tolist()
    assert any(t % 3600 for t in fr["t"])
    np.testing.assert_array_equal((fr["status"] > 2).astype(np.int8), ref["status"])
    tn = np.asarray(net.tank_node)
    junc = np.asarray(net.node_type) == 0
    assert np.abs(fr["tank_head"] - ref["head_ft"][:, tn]).max() < 1e-7
    assert np.abs(fr["head"][:, junc] - ref["head_ft"][:, junc]).max() < 1e-7
    assert np.abs(fr["flow"] - ref["flow_int_cfs"]).max() < 1e-7
    o = EpsOracle(net).run(inp["demand"], rh, np.asarray(net.tank_h0)[None], accuracy=1e-9)[0]
    assert np.abs(fr["head"] - np.stack(o["head"])).max() <= HEAD_ATOL_FT
    assert np.abs(fr["tank_head"] - np.stack(o["tank_head"])).max() <= HEAD_ATOL_FT


def test_eps_forward_matches_oracle(setup):
    from wdsgpu_b200.eps import eps_solve
    net, s, dem, rh, th0 = setup
    out = eps_solve(s, dem, rh, th0, accuracy=1e-9)
    runs = EpsOracle(net).run(dem, rh, th0, accuracy=1e-9)
    for b, fr_o in enumerate(runs):
        fr = _frames(out, b)
        assert fr["t"] == fr_o["t"]
        assert np.abs(fr["tank_head"] - np.stack(fr_o["tank_head"])).max() <= HEAD_ATOL_FT
        assert np.abs(fr["head"] - np.stack(fr_o["head"])).max() <= HEAD_ATOL_FT
        assert np.abs(fr["flow"] - np.stack(fr_o["flow"])).max() <= 1e-9


def test_eps_gradients_match_oracle_adjoint(setup):
    from wdsgpu_b200.eps import eps_solve
    net, s, dem, rh, th0 = setup
    P, B = dem.shape[:2]
    dev = s.device
    sens = np.flatnonzero(np.asarray(net.node_type) == 0)[::5]
    wq = np.random.default_rng(2).normal(size=net.L)
    D = torch.tensor(dem, device=dev, requires_grad=True)
    H0 = torch.tensor(th0, device=dev, requires_grad=True)
    R = torch.tensor(np.asarray(net.r_hw), device=dev, requires_grad=True)
    out = eps_solve(s, D, torch.tensor(rh, device=dev), H0, r_hw=R, accuracy=1e-10)
    loss = ((out["head"][:, :, sens] ** 2).sum() + (out["tank_head"][-1] ** 2).sum()
            + (out["flow"] * torch.tensor(wq, device=dev)).sum())
    loss.backward()
    assert bool(out["valid"].all())            # no tank event: the frames line up
    eo = EpsOracle(net)
    runs = eo.run(dem, rh, th0, accuracy=1e-10)
    mask = np.isin(np.arange(net.N), sens)
    gH = [[np.where(mask, 2.0 * h, 0.0) for h in fr["head"]] for fr in runs]
    gQ = [[wq for _ in fr["flow"]] for fr in runs]
    gE = [[np.zeros(net.N) for _ in fr["flow"]] for fr in runs]
    gT = [[np.zeros(len(net.tank_node)) for _ in fr["flow"]] for fr in runs]
    for fr, g in zip(runs, gT):
        g[-1] = 2.0 * fr["tank_head"][-1]
    g_dem, _, g_h0, _, g_r = eo.backward(runs, gH, gQ, gE, gT, P=P)
    for a, b in ((D.grad, g_dem), (H0.grad, g_h0), (R.grad, g_r.sum(0))):
        a = a.cpu().numpy()
        assert np.abs(a - b).max() <= GRAD_RTOL * np.abs(b).max(), np.abs(a - b).max()


def test_eps_tank_gradient_central_difference(setup):
    """dL/d(initial tank head) of the GPU path against its own central
    difference (small step: the tank pathway is strongly curved)."""
    from wdsgpu_b200.eps import eps_solve
    net, s, dem, rh, th0 = setup
    dev = s.device
    dem3 = dem[:3]

    def run(h0, grad=False):
        H0 = torch.tensor(h0, device=dev, requires_grad=grad)
        out = eps_solve(s, dem3, rh, H0, accuracy=1e-12)
        return (out["tank_head"][-1] ** 2).sum(), H0

    loss, H0 = run(th0, True)
    loss.backward()
    g = H0.grad.cpu().numpy()
    eps = 1e-5
    for b, i in ((0, 0), (2, 1)):
        hp, hm = th0.copy(), th0.copy()
        hp[b, i] += eps
        hm[b, i] -= eps
        fd = (float(run(hp)[0]) - float(run(hm)[0])) / (2 * eps)
        assert abs(g[b, i] - fd) <= 1e-6 * abs(fd), (g[b, i], fd)
