"""Large-network layout (tables and scenario state in global memory, one CTA
per scenario): bitwise equal to the shared-memory layout where both apply,
and correct against the oracle on a network too large for shared memory."""
import numpy as np
import pytest
import torch

from oracle.gga import Model
from wdsgpu_b200 import synth
from wdsgpu_b200.solver import GGASolver
from wdsgpu_b200.autodiff import implicit_solve

pytestmark = pytest.mark.gpu

POLISHED_HEAD_ATOL_FT = 1e-9 / 0.3048


def _run(net, cuda, layout, d, rh, B):
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    s.sm100_layout = layout
    ke = s.node_ke_default.unsqueeze(0).contiguous()
    r = s.r_hw.unsqueeze(0).contiguous()
    o = s.run(torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda), ke, r, B, 200,
              1e-6, True, 3)
    torch.cuda.synchronize()
    return s, o


@pytest.mark.parametrize("which", ["config2", "feature"])
def test_global_layout_equals_shared_layout_bitwise(cuda, which):
    net = synth.config2_network() if which == "config2" else synth.feature_network()
    B = 6
    d, rh = synth.config2_scenarios(net, B, seed=21, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    s1, a = _run(net, cuda, "shared", d, rh, B)
    s2, b = _run(net, cuda, "global", d, rh, B)
    assert s1.plan_stats(B)["smem_bytes"] > 0 and s2.plan_stats(B)["smem_bytes"] == 0
    for k in ("head", "flow", "emit", "status", "iters", "info"):
        assert torch.equal(a[k], b[k]), k
    # adjoint on the kept terminal state
    for s in (s1, s2):
        D = torch.tensor(d, device=cuda, requires_grad=True)
        h = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-6)[0]
        (h ** 2).sum().backward()
        s._g = D.grad.clone()
    assert torch.equal(s1._g, s2._g)


def test_network_beyond_shared_memory_matches_oracle(cuda):
    """3000 junctions / 3600 pipes: the plan falls back to the global layout;
    iterations exact, polished heads within 1e-9 m, gradients within 1e-6."""
    net = synth.config3_networks()[3]
    B = 2
    d, rh = synth.config2_scenarios(net, B, seed=5, sigma=0.3)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    assert s.plan_stats(B)["smem_bytes"] == 0                 # global layout chosen
    D = torch.tensor(d, device=cuda, requires_grad=True)
    sens = synth.sensor_nodes(net, 30)
    h, q, e = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-9)
    (h[:, sens] ** 2).sum().backward()
    m = Model(net)
    o, st = m.implicit(d, rh, accuracy=1e-9)
    assert np.abs(h.detach().cpu().numpy() - o["head_ft"]).max() <= POLISHED_HEAD_ATOL_FT
    assert np.abs(q.detach().cpu().numpy() - o["flow_cfs"]).max() <= 1e-9
    gH = np.zeros((B, net.N))
    gH[:, sens] = 2.0 * o["head_ft"][:, sens]
    gd = m.backward(st, gH, np.zeros((B, net.L)), np.zeros((B, net.N)))[0]
    g = D.grad.cpu().numpy()
    assert np.abs(g - gd).max() <= 1e-6 * np.abs(gd).max()
    f = s.solve(d, rh, status_machine=True, accuracy=1e-6)
    ref = m.solve(d, rh, accuracy=1e-6, status_machine=True)
    assert np.array_equal(f["iters"].cpu().numpy(), ref["iters"])
