"""Extended-period run at the full workload size (about 20 000 junctions,
23 000 pipes, 4 pumps, 3 tanks; the large-network layout).  No dense oracle
reaches this size, so the checks are size-independent: mass balance at every
junction of every frame, the tank-volume identity between frames, and central
differences of the gradients through time."""
import numpy as np
import pytest
import torch

from wdsgpu_b200 import synth
from wdsgpu_b200.eps import eps_solve, tank_links
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def big(cuda):
    net0 = synth.config5_network()
    pre = synth.tanks_as_junctions(net0)
    s0 = GGASolver(pre, device=cuda, dense_status_machine=True)
    d = pre.demand_cfs_at(0)[None] * synth.diurnal(0.0)
    o = s0.solve(d, np.nan_to_num(pre.fixed_head_ft_at(0))[None], status_machine=True,
                 accuracy=1e-8)
    ctr = o["head_ft"][0].cpu().numpy()[np.asarray(net0.tank_node)]
    net = synth.config5_network(tank_center_ft=ctr)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    return net, s


def test_eps_full_size_mass_balance_and_tank_identity(big):
    net, s = big
    T, B = 3, 4
    dem = synth.eps_demands(net, T, B, seed=2)
    out = eps_solve(s, dem, accuracy=1e-10)
    assert s.plan_stats(B)["smem_bytes"] == 0           # global layout
    q = out["flow"].cpu().numpy()
    n1, n2 = np.asarray(net.link_n1), np.asarray(net.link_n2)
    junc = np.flatnonzero(np.asarray(net.node_type) == 0)
    for t in range(T):
        inflow = np.zeros((B, net.N))
        for b in range(B):
            np.add.at(inflow[b], n2, q[t, b])
            np.add.at(inflow[b], n1, -q[t, b])
        resid = inflow[:, junc] - dem[t][:, junc]
        assert np.abs(resid).max() <= 1e-8 * np.abs(dem[t]).max() * 100, np.abs(resid).max()
    # tank identity: V(next frame) - V(frame) = step * net inflow (no clamp here)
    assert bool(out["valid"].all())
    ks, js, sg = tank_links(s)
    area = np.asarray(net.tank_area)
    th = out["tank_head"].cpu().numpy()
    ts = out["t_sec"].cpu().numpy()
    for t in range(T - 1):
        qnet = np.zeros((B, len(area)))
        for k, j, sgn in zip(ks, js, sg):
            qnet[:, j] += sgn * q[t, :, k]
        dv = (th[t + 1] - th[t]) * area
        step = (ts[t + 1] - ts[t]).astype(np.float64)[:, None]
        assert np.abs(dv - step * qnet).max() <= 1e-6 * max(1.0, np.abs(dv).max())


def test_eps_full_size_gradients_central_difference(big):
    net, s = big
    T, B = 3, 2
    dev = s.device
    dem = synth.eps_demands(net, T, B, seed=4)
    j = int(np.flatnonzero(np.asarray(net.node_type) == 0)[12345])
    sens = np.arange(0, net.N, 97)

    def loss_of(d, h0):
        out = eps_solve(s, d, tank_h0=h0, accuracy=1e-12)
        return ((out["head"][:, :, sens] ** 2).sum() + (out["tank_head"][-1] ** 2).sum())

    h0 = np.broadcast_to(np.asarray(net.tank_h0), (B, 3)).copy()
    D = torch.tensor(dem, device=dev, requires_grad=True)
    H0 = torch.tensor(h0, device=dev, requires_grad=True)
    loss_of(D, H0).backward()
    eps = 1e-3 * dem[0, 1, j]
    dp, dm = dem.copy(), dem.copy()
    dp[0, 1, j] += eps
    dm[0, 1, j] -= eps
    fd = (float(loss_of(dp, h0)) - float(loss_of(dm, h0))) / (2 * eps)
    assert abs(float(D.grad[0, 1, j]) - fd) <= 1e-5 * abs(fd), (float(D.grad[0, 1, j]), fd)
    eps = 1e-5
    hp, hm = h0.copy(), h0.copy()
    hp[0, 2] += eps
    hm[0, 2] -= eps
    fd = (float(loss_of(dem, hp)) - float(loss_of(dem, hm))) / (2 * eps)
    assert abs(float(H0.grad[0, 2]) - fd) <= 1e-5 * abs(fd), (float(H0.grad[0, 2]), fd)
