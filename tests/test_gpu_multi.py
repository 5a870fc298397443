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


def test_multi_matches_reference_goldens(cuda):
    """The mixed-size workload's 100-junction and 79-TCV networks and the
    782-junction network in one multi-plan launch, against the reference's own
    outputs (tests/golden/cfg3_small.npz, cfg3_tcv.npz, cfg2.npz): iterations
    and statuses exact, polished heads within 1e-9 m, gradients w.r.t.
    demand, Ke and r within 1e-6 relative."""
    from tests.golden.load import load
    cases = [load(t) for t in ("cfg3_small", "cfg3_tcv", "cfg2")]
    solvers = [GGASolver(net, device=cuda, dense_status_machine=True) for net, _, _ in cases]
    acc = float(cases[0][1]["accuracy"])
    assert all(float(inp["accuracy"]) == acc for _, inp, _ in cases)
    fw = solve_multi(solvers, [inp["demand"] for _, inp, _ in cases],
                     [inp["res_head"] for _, inp, _ in cases],
                     kes=[inp["ke"] for _, inp, _ in cases], accuracy=acc, status_machine=True)
    for (net, inp, ref), r in zip(cases, fw):
        np.testing.assert_array_equal(r["iters"].cpu().numpy(), ref["fwd_iters"])
        np.testing.assert_array_equal(r["status"].cpu().numpy(), ref["fwd_status"])
        assert np.abs(r["head_ft"].cpu().numpy() - ref["fwd_head"]).max() < 1e-4
    Ds = [torch.tensor(inp["demand"], device=cuda, requires_grad=True) for _, inp, _ in cases]
    Ks = [torch.tensor(inp["ke"][0], device=cuda, requires_grad=True) for _, inp, _ in cases]
    Rs = [torch.tensor(np.asarray(net.r_hw), device=cuda, requires_grad=True)
          for net, _, _ in cases]
    outs = implicit_solve_multi(solvers, Ds, [torch.tensor(inp["res_head"], device=cuda)
                                              for _, inp, _ in cases],
                                kes=Ks, r_hws=Rs, accuracy=acc)
    loss = sum((h[:, inp["sensors"]] ** 2).sum() for (h, _, _), (_, inp, _) in zip(outs, cases))
    loss.backward()

    def rel(a, b):
        return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))

    for (net, inp, ref), (h, q, e), D, K, R in zip(cases, outs, Ds, Ks, Rs):
        assert np.abs(h.detach().cpu().numpy() - ref["imp_head"]).max() < 1e-9 / 0.3048
        assert np.abs(q.detach().cpu().numpy() - ref["imp_flow"]).max() < 1e-9
        assert rel(D.grad.cpu().numpy(), ref["grad_demand"]) < 1e-6
        assert rel(R.grad.cpu().numpy(), ref["grad_r"]) < 1e-6
        if np.abs(ref["grad_ke"]).max() > 0:
            assert rel(K.grad.cpu().numpy(), ref["grad_ke"]) < 1e-6
