"""Extended-period run on the GPU (wdsgpu_b200.eps.eps_solve) against the
oracle composition (oracle/eps.py, itself pinned to the reference's
EpsDriver): trajectory, adjoint through time, and central differences."""
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


@pytest.fixture(scope="module")
def setup(cuda):
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("eps_ref")
    T, B = 4, 3
    rng = np.random.default_rng(8)
    dem = inp["demand"][:T, :1].repeat(B, 1) * rng.uniform(0.85, 1.15, (T, B, net.N))
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), (B, net.N)).copy()
    th0 = np.broadcast_to(np.asarray(net.tank_h0), (B, len(net.tank_node))).copy()
    th0 = th0 + rng.uniform(-0.5, 0.5, th0.shape)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    return net, s, dem, rh, th0


def test_eps_forward_matches_oracle(setup):
    from wdsgpu_b200.eps import eps_solve
    net, s, dem, rh, th0 = setup
    out = eps_solve(s, dem, rh, th0, accuracy=1e-9)
    ref = EpsOracle(net).run(dem, rh, th0, accuracy=1e-9)
    assert np.abs(out["tank_head"].cpu().numpy() - ref["tank_head"]).max() <= HEAD_ATOL_FT
    assert np.abs(out["head"].cpu().numpy() - ref["head"]).max() <= HEAD_ATOL_FT
    assert np.abs(out["flow"].cpu().numpy() - ref["flow"]).max() <= 1e-9


def test_eps_gradients_match_oracle_adjoint(setup):
    from wdsgpu_b200.eps import eps_solve
    net, s, dem, rh, th0 = setup
    T, B = dem.shape[:2]
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
    eo = EpsOracle(net)
    run = eo.run(dem, rh, th0, accuracy=1e-10)
    gH = np.zeros((T, B, net.N))
    gH[:, :, sens] = 2.0 * run["head"][:, :, sens]
    gT = np.zeros((T + 1, B, len(net.tank_node)))
    gT[T] = 2.0 * run["tank_head"][T]
    g_dem, _, g_h0, _, g_r = eo.backward(run, gH, np.broadcast_to(wq, (T, B, net.L)),
                                         np.zeros((T, B, net.N)), gT)
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
