"""The large-batch workload: B = 16384 scenarios of the 782-junction network
in one persistent launch (111 rounds of the 148 CTAs), FP64 factor.  Every
scenario converges, a sample from the first, middle and last rounds agrees
with the oracle (polished heads within 1e-9 m, demand gradients within 1e-6
relative), and mass balances at every junction of every scenario."""
import numpy as np
import pytest
import torch

from oracle.gga import Model
from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu

B = 16384


def test_b16384_config2_against_oracle_sample(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = synth.config2_scenarios(net, B, seed=16384)
    D = torch.tensor(d, device=cuda, requires_grad=True)
    h, q, e = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-6)
    sens = synth.sensor_nodes(net, 30)
    (h[:, sens] ** 2).sum().backward()
    assert torch.isfinite(D.grad).all()
    pick = np.array([0, 147, 443, 8191, 8192 + 77, 16383 - 148, 16383])
    m = Model(net)
    out, st = m.implicit(d[pick], rh[pick], accuracy=1e-6)
    hn = h.detach().cpu().numpy()
    assert np.abs(hn[pick] - out["head_ft"]).max() < 1e-9 / 0.3048
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd = m.backward(st, gH, np.zeros_like(out["flow_cfs"]), np.zeros_like(out["emitter_cfs"]))[0]
    g = D.grad.cpu().numpy()[pick]
    assert float(np.abs(g - gd).max() / np.abs(gd).max()) < 1e-6
    qn = q.detach().cpu().numpy()
    n1, n2 = np.asarray(net.link_n1), np.asarray(net.link_n2)
    junc = np.flatnonzero(np.asarray(net.node_type) == 0)
    bal = np.zeros((B, net.N))
    np.add.at(bal.T, n2, qn.T)
    np.add.at(bal.T, n1, -qn.T)
    bal -= d + e.detach().cpu().numpy()
    assert np.abs(bal[:, junc]).max() < 1e-9
