"""Unrolled-K differentiation on the B200 route (solve_unrolled): the
recording forward and wds_unrolled_adjoint against the reference's
solve_unrolled and its autograd gradients (fixture
tests/golden/unrolled_ref.npz, and unrolled_warm_ref.npz for warm starts and
frozen statuses) and against the oracle's reverse pass on unseen scenarios,
other K and per-scenario statuses."""
import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.gga import Model  # noqa: E402
from oracle.unrolled import Unrolled  # noqa: E402
from test_unrolled_oracle import unrolled_loss_adjoints  # noqa: E402

pytestmark = pytest.mark.gpu


def _gpu_run(s, net, inp, d, rh, ke, K, cuda, **warm):
    from wdsgpu_b200.autodiff import solve_unrolled
    D = torch.tensor(d, device=cuda).requires_grad_(True)
    RH = torch.tensor(rh, device=cuda).requires_grad_(True)
    KE = torch.tensor(ke, device=cuda).requires_grad_(True)
    R = torch.tensor(np.asarray(net.r_hw, dtype=np.float64), device=cuda).requires_grad_(True)
    out = solve_unrolled(s, D, RH, ke=KE, r_hw=R, K=K, **warm)
    h, q, e = out["head_ft"], out["flow_cfs"], out["emitter_cfs"]
    sens = torch.as_tensor(np.asarray(inp["sensors"]), device=cuda)
    pl = torch.as_tensor(np.asarray(net.pump_link), device=cuda)
    emn = torch.as_tensor(np.flatnonzero(np.asarray(net.node_ke) > 0), device=cuda)
    ((h[:, sens] ** 2).sum() + (q[:, pl] ** 2).sum() + (e[:, emn] ** 2).sum()).backward()
    o = {k: v.detach().cpu().numpy() for k, v in out.items()}
    g = dict(g_demand=D.grad.cpu().numpy(), g_res_head=RH.grad.cpu().numpy(),
             g_ke=KE.grad.cpu().numpy(), g_rhw=R.grad.cpu().numpy())
    return o, g


def test_unrolled_matches_reference(cuda):
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load("unrolled_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    o, g = _gpu_run(s, net, inp, inp["demand"], inp["res_head"], inp["ke"], int(inp["K"]), cuda)
    assert np.abs(o["head_ft"] - ref["head"]).max() < 1e-4      # unconverged K-iteration state
    assert np.abs(o["flow_cfs"] - ref["flow"]).max() < 1e-6
    junc = np.asarray(net.node_type) == 0
    for key, cols in (("g_demand", junc), ("g_res_head", ~junc), ("g_ke", junc),
                      ("g_rhw", slice(None))):
        G, R = g[key][..., cols], ref[key][..., cols]
        assert np.abs(G - R).max() <= 1e-6 * np.abs(R).max(), (key, np.abs(G - R).max())


@pytest.mark.parametrize("K", [5, 12])
def test_unrolled_against_oracle(cuda, K):
    from wdsgpu_b200 import synth
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("unrolled_ref")
    d, _ = synth.config2_scenarios(net, 5, seed=83, sigma=0.35)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    ke = np.broadcast_to(np.asarray(net.node_ke, dtype=np.float64), d.shape).copy()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    o, g = _gpu_run(s, net, inp, d, rh, ke, K, cuda)
    u = Unrolled(Model(net))
    oo, st = u.forward(d, rh, ke=ke, K=K)
    assert np.abs(o["head_ft"] - oo["head_ft"]).max() < 1e-4
    gd, grh, gke, gr = u.backward(st, *unrolled_loss_adjoints(net, inp, oo)[:3])
    junc = np.asarray(net.node_type) == 0
    for G, R, cols in ((g["g_demand"], gd, junc), (g["g_res_head"], grh, ~junc),
                       (g["g_ke"], gke, junc), (g["g_rhw"], gr.sum(0), slice(None))):
        assert np.abs(G[..., cols] - R[..., cols]).max() <= 1e-6 * np.abs(R[..., cols]).max()


def test_unrolled_warm_matches_reference(cuda):
    """Warm start q0 [B,L] / e0 [B,N] and frozen statuses [L] against the
    reference's solve_unrolled (fixture unrolled_warm_ref.npz)."""
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load("unrolled_warm_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    o, g = _gpu_run(s, net, inp, inp["demand"], inp["res_head"], inp["ke"], int(inp["K"]), cuda,
                    q0=torch.tensor(inp["q0"], device=cuda),
                    e0=torch.tensor(inp["e0"], device=cuda), status=inp["status"])
    assert np.abs(o["head_ft"] - ref["head"]).max() < 1e-4
    assert np.abs(o["flow_cfs"] - ref["flow"]).max() < 1e-6
    assert np.abs(o["emitter_cfs"] - ref["emitter"]).max() < 1e-6
    junc = np.asarray(net.node_type) == 0
    for key, cols in (("g_demand", junc), ("g_res_head", ~junc), ("g_ke", junc),
                      ("g_rhw", slice(None))):
        G, R = g[key][..., cols], ref[key][..., cols]
        assert np.abs(G - R).max() <= 1e-6 * np.abs(R).max(), (key, np.abs(G - R).max())


def test_unrolled_frozen_status_per_scenario(cuda):
    """Per-scenario frozen statuses [B,L] without q0: the initial flows follow
    the statuses (closed links QZERO); recording forward and reverse pass
    against the oracle with the same start."""
    from wdsgpu_b200 import synth
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("unrolled_warm_ref")
    d, _ = synth.config2_scenarios(net, 4, seed=29, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    ke = np.broadcast_to(np.asarray(net.node_ke, dtype=np.float64), d.shape).copy()
    S = np.broadcast_to(np.asarray(inp["status"], dtype=np.int8), (4, net.L)).copy()
    pipes = np.flatnonzero(np.asarray(net.link_type) == 1)
    S[1, pipes[5]] = 2                      # another pipe closed in scenario 1
    S[3, pipes[9]] = 2
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    o, g = _gpu_run(s, net, inp, d, rh, ke, 7, cuda, status=S)
    u = Unrolled(Model(net))
    q0 = np.where(S <= 2, 1e-6, s._q_open)
    oo, st = u.forward(d, rh, ke=ke, K=7, S=S, q0=q0)
    assert np.abs(o["head_ft"] - oo["head_ft"]).max() < 1e-4
    assert np.abs(o["flow_cfs"] - oo["flow_cfs"]).max() < 1e-6
    gd, grh, gke, gr = u.backward(st, *unrolled_loss_adjoints(net, inp, oo)[:3])
    junc = np.asarray(net.node_type) == 0
    for G, R, cols in ((g["g_demand"], gd, junc), (g["g_res_head"], grh, ~junc),
                       (g["g_ke"], gke, junc), (g["g_rhw"], gr.sum(0), slice(None))):
        assert np.abs(G[..., cols] - R[..., cols]).max() <= 1e-6 * np.abs(R[..., cols]).max()


def test_unrolled_refuses_control_valves(cuda):
    from wdsgpu_b200 import synth
    from wdsgpu_b200.autodiff import solve_unrolled
    from wdsgpu_b200.solver import GGASolver
    net = synth.config2_network()                 # PRVs with a setting
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    with pytest.raises(NotImplementedError):
        solve_unrolled(s, net.demand_cfs_at(0), net.reservoir_head_ft_at(0), K=5)


def test_unrolled_grad_health(cuda):
    """The health probe's rel_K is the relative change of the unrolled
    gradient between K + dK and K + 2 dK, and the verdict follows the
    reference's thresholds."""
    from wdsgpu_b200.autodiff import (GRAD_HEALTH_COND, GRAD_HEALTH_OK, VERDICT_COND,
                                      VERDICT_NO, VERDICT_OK, solve_unrolled,
                                      unrolled_grad_health)
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("unrolled_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = inp["demand"][:2], inp["res_head"][:2]
    rep = unrolled_grad_health(s, d, rh, K=8, dK=4, vs_implicit=True)
    W = torch.as_tensor(np.random.default_rng(0).normal(0, 1, (2, net.N)), device=cuda)

    def grad(K):
        D = torch.tensor(d, device=cuda).requires_grad_(True)
        g, = torch.autograd.grad((solve_unrolled(s, D, torch.tensor(rh, device=cuda), K=K)
                                  ["head_ft"] * W).sum(), D)
        return g
    g1, g2 = grad(12), grad(16)
    rel = float((g1 - g2).abs().max() / torch.max(g1.abs().max(), g2.abs().max()))
    assert abs(rep["rel_K"] - rel) <= 1e-12 + 1e-9 * rel
    want = (VERDICT_OK if rep["rel_K"] < GRAD_HEALTH_OK and rep["rel_implicit"] < 1e-6 else
            VERDICT_COND if rep["rel_K"] < GRAD_HEALTH_COND and rep["rel_implicit"] < 1e-3 else
            VERDICT_NO)
    assert rep["verdict"] == want and rep["K"] == 8 and rep["rel_implicit"] is not None
