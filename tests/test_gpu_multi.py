"""Networks of different sizes in one launch (the mixed-size workload: 100,
542 with 79 TCVs, 782 with 3 PRVs, and 3000 junctions, the last one too large
for shared memory): per network the results of one multi-plan launch equal
those of that network's own launch, bitwise, for the forward and for the
gradients."""
import numpy as np
import pytest
import torch

from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.multi import implicit_solve_multi, solve_multi
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed(cuda):
    nets = synth.config3_networks()
    rng = np.random.default_rng(3)
    counts = np.bincount(rng.integers(0, 4, 64), minlength=4)   # instances per network
    data = []
    for i, (net, B) in enumerate(zip(nets, counts)):
        d, _ = synth.config2_scenarios(net, int(B), seed=40 + i, sigma=0.3)
        rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
        data.append((net, d, rh))
    return data


def _solvers(data, cuda):
    return [GGASolver(net, device=cuda, dense_status_machine=True) for net, _, _ in data]


def test_multi_forward_equals_single_launches(mixed, cuda):
    a = _solvers(mixed, cuda)
    b = _solvers(mixed, cuda)
    assert b[3].plan_stats(8)["smem_bytes"] == 0               # large network: global layout
    res = solve_multi(a, [d for _, d, _ in mixed], [rh for _, _, rh in mixed],
                      accuracy=1e-6, status_machine=True)
    for s, (net, d, rh), r in zip(b, mixed, res):
        one = s.solve(d, rh, status_machine=True, accuracy=1e-6)
        for k in ("head_ft", "flow_cfs", "iters", "status", "converged"):
            assert torch.equal(r[k], one[k]), k


def test_multi_implicit_and_adjoint_equal_single_launches(mixed, cuda):
    a = _solvers(mixed, cuda)
    b = _solvers(mixed, cuda)
    Ds = [torch.tensor(d, device=cuda, requires_grad=True) for _, d, _ in mixed]
    outs = implicit_solve_multi(a, Ds, [torch.tensor(rh, device=cuda) for _, _, rh in mixed],
                                accuracy=1e-6)
    loss = sum((h ** 2).sum() + (q ** 2).sum() for h, q, _ in outs)
    loss.backward()
    for s, (net, d, rh), D, (h, q, e) in zip(b, mixed, Ds, outs):
        D1 = torch.tensor(d, device=cuda, requires_grad=True)
        h1, q1, e1 = implicit_solve(s, D1, torch.tensor(rh, device=cuda), accuracy=1e-6)
        ((h1 ** 2).sum() + (q1 ** 2).sum()).backward()
        assert torch.equal(h, h1) and torch.equal(q, q1)
        assert torch.equal(D.grad, D1.grad)
