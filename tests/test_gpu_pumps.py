"""Pump-parameter gradients on the B200 route: implicit_solve(speed=,
pump_h0=, pump_r=) through wds_forward (the call's pump rows) and
wds_adjoint_pumps, against the reference's CPU adjoint with pump theta
(fixture tests/golden/pump_ref.npz, dgga/autodiff.py:609-756) and against the
oracle for per-scenario rows, zero speed and the pumpstatus shut-off at the
call's speed."""
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
from test_pump_oracle import pump_loss_grads  # noqa: E402

pytestmark = pytest.mark.gpu


def _gpu_loss_grads(s, net, inp, th, cuda, per_row=False):
    from wdsgpu_b200.autodiff import implicit_solve
    B = inp["demand"].shape[0]
    pl = np.asarray(net.pump_link)
    pn2 = np.asarray(net.link_n2)[pl]
    ts = []
    for v in th:
        t = torch.tensor(np.asarray(v), dtype=torch.float64, device=cuda)
        if per_row and t.dim() == 1:
            t = t.unsqueeze(0).expand(B, -1).contiguous()
        ts.append(t.requires_grad_(True))
    D = torch.tensor(inp["demand"], device=cuda).requires_grad_(True)
    RH = torch.tensor(np.nan_to_num(inp["res_head"]), device=cuda).requires_grad_(True)
    h, q, e = implicit_solve(s, D, RH, ke=torch.tensor(inp["ke"], device=cuda), accuracy=1e-7,
                             speed=ts[0], pump_h0=ts[1], pump_r=ts[2])
    sens = torch.as_tensor(np.asarray(inp["sensors"]), device=cuda)
    loss = (h[:, sens] ** 2).sum() + (h[:, torch.as_tensor(pn2, device=cuda)] ** 2).sum() \
        + (q[:, torch.as_tensor(pl, device=cuda)] ** 2).sum()
    loss.backward()
    _gpu_loss_grads.g_res_head = RH.grad.cpu().numpy()
    return h.detach().cpu().numpy(), q.detach().cpu().numpy(), D.grad.cpu().numpy(), \
        [t.grad.cpu().numpy() for t in ts]


@pytest.mark.parametrize("case", ["pump_ref", "chp_ref"])
def test_pump_theta_matches_reference(cuda, case):
    """pump_ref: all four pump kinds at moved parameters; chp_ref: a
    constant-HP pump on its CBIG clamp branch (exact Jacobian by the Woodbury
    correction on the kept factor).  In chp_ref the dead-end junction hangs on
    the pump's 1/CBIG conductance, so the reduced system has a condition
    number near 1e10 and the gradient at that junction (4e12) agrees to about
    1e-8 relative; elsewhere to 1e-10."""
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load(case)
    tol = 1e-8 if case == "pump_ref" else 1e-7
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    th = (inp["speed"], inp["pump_h0"], inp["pump_r"])
    # [L] rows shared by the batch: the batch-summed gradient, as the reference
    h, q, gd, g = _gpu_loss_grads(s, net, inp, th, cuda)
    assert np.abs(h - ref["head"]).max() <= 1e-9 * max(np.abs(ref["head"]).max(), 1e3)
    assert np.abs(gd - ref["g_demand"]).max() <= tol * np.abs(ref["g_demand"]).max()
    grh = _gpu_loss_grads.g_res_head
    fixed = np.asarray(net.node_type) != 0
    R = ref["g_res_head"][:, fixed]
    assert np.abs(grh[:, fixed] - R).max() <= tol * np.abs(R).max()
    for gi, key in zip(g, ("g_speed", "g_h0", "g_r")):
        R = ref[key].sum(0)
        assert np.abs(gi - R).max() <= tol * np.abs(R).max(), (key, np.abs(gi - R).max())
    # [B,L] rows: one gradient row per scenario
    _, _, _, g = _gpu_loss_grads(s, net, inp, th, cuda, per_row=True)
    for gi, key in zip(g, ("g_speed", "g_h0", "g_r")):
        R = ref[key]
        assert gi.shape == R.shape
        assert np.abs(gi - R).max() <= tol * np.abs(R).max(), (key, np.abs(gi - R).max())


def test_network_values_are_the_default(cuda):
    """Passing the network's own speeds / coefficients changes nothing, bit
    for bit (the pumpstatus shut-off w^2 Hmax is formed as the planner does)."""
    from wdsgpu_b200.autodiff import implicit_solve
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("pump_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d = torch.tensor(inp["demand"], device=cuda)
    rh = torch.tensor(inp["res_head"], device=cuda)
    a = implicit_solve(s, d, rh, accuracy=1e-7)
    b = implicit_solve(s, d, rh, accuracy=1e-7, speed=s.init_setting,
                       pump_h0=s._tables["pump_h0"], pump_r=s._tables["pump_r"])
    for x, y in zip(a, b):
        assert torch.equal(x, y)


def _check_against_oracle(net, inp, th_rows, h, q, gd, g):
    B = inp["demand"].shape[0]
    for b in range(B):
        m = Model(net).with_pumps(*(t[b] for t in th_rows))
        one = dict(demand=inp["demand"][b:b + 1], res_head=inp["res_head"][b:b + 1],
                   ke=inp["ke"], sensors=inp["sensors"])
        out, _, go = pump_loss_grads(m, net, one)
        assert np.abs(h[b] - out["head_ft"][0]).max() < 1e-8
        assert np.abs(q[b] - out["flow_cfs"][0]).max() < 1e-8
        assert np.abs(gd[b] - go[0][0]).max() <= 1e-8 * np.abs(go[0]).max()
        for gi, oi in zip(g, go[4:]):
            assert np.abs(gi[b] - oi[0]).max() <= 1e-8 * max(np.abs(oi).max(), 1.0)


def test_per_scenario_speeds_against_oracle(cuda):
    """Different pump speeds per scenario, with the supply pump and the
    constant-HP pump stopped in one scenario each (closed branch)."""
    from wdsgpu_b200.solver import GGASolver
    net, inp, _ = load("pump_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    pl = np.asarray(net.pump_link)
    B = inp["demand"].shape[0]
    sp = np.tile(inp["speed"], (B, 1))
    sp[0, pl[0]] = 0.0            # power-function supply pump stopped: the tank feeds
    sp[1, pl[3]] = 0.0            # constant-HP pump stopped
    sp[2, pl[0]] = 1.08
    th = (sp, np.tile(inp["pump_h0"], (B, 1)), np.tile(inp["pump_r"], (B, 1)))
    h, q, gd, g = _gpu_loss_grads(s, net, inp, th, cuda)
    _check_against_oracle(net, inp, th, h, q, gd, g)
    assert g[0][0, pl[0]] == 0.0 and g[0][1, pl[3]] == 0.0


def test_pumpstatus_shutoff_at_call_speed(cuda):
    """Lifting pumps (tanks above a low reservoir): at speed 0.8 the first
    pump's shut-off head w^2 Hmax falls below the lift and pumpstatus takes it
    to XHEAD; the status machine follows the call's speed per scenario."""
    from wdsgpu_b200 import synth
    from wdsgpu_b200.solver import GGASolver
    net = synth.eps_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    pl = np.asarray(net.pump_link)
    d0 = net.demand_cfs_at(0)
    d = np.stack([d0 * f for f in (1.0, 0.9, 1.1)])
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    inp = dict(demand=d, res_head=rh, ke=np.asarray(net.node_ke, dtype=np.float64),
               sensors=synth.sensor_nodes(net, 6))
    sp = np.tile(s.init_setting, (3, 1))
    sp[1, pl[0]] = 0.8
    sp[2, pl[1]] = 1.1
    th = (sp, np.tile(s._tables["pump_h0"], (3, 1)), np.tile(s._tables["pump_r"], (3, 1)))
    h, q, gd, g = _gpu_loss_grads(s, net, inp, th, cuda)
    _check_against_oracle(net, inp, th, h, q, gd, g)
    assert abs(q[1, pl[0]]) < 1e-5 and abs(q[0, pl[0]]) > 1e-3
    assert g[0][1, pl[0]] == 0.0 and g[0][0, pl[0]] != 0.0


def test_clamp_branch_in_multi_and_eps_routes(cuda):
    """The constant-HP clamp-branch correction in the multi-plan launch (the
    same gradients as one implicit_solve per network) and in the
    extended-period adjoint (the oracle's adjoint through time, whose steps use
    the exact clamp Jacobian)."""
    from wdsgpu_b200 import synth
    from wdsgpu_b200.autodiff import implicit_solve
    from wdsgpu_b200.eps import eps_solve
    from wdsgpu_b200.multi import implicit_solve_multi
    from wdsgpu_b200.solver import GGASolver
    from oracle.eps import EpsOracle
    nets = [load("chp_ref"), load("pump_ref")]
    solvers = [GGASolver(net, device=cuda, dense_status_machine=True) for net, _, _ in nets]
    Ds = [torch.tensor(inp["demand"], device=cuda).requires_grad_(True) for _, inp, _ in nets]
    RHs = [torch.tensor(np.nan_to_num(inp["res_head"]), device=cuda) for _, inp, _ in nets]
    outs = implicit_solve_multi(solvers, Ds, RHs, accuracy=1e-7)
    sum((h ** 2).sum() for h, _, _ in outs).backward()
    for s, D, RH in zip(solvers, Ds, RHs):
        D1 = D.detach().clone().requires_grad_(True)
        (implicit_solve(s, D1, RH, accuracy=1e-7)[0] ** 2).sum().backward()
        G, R = D.grad.cpu().numpy(), D1.grad.cpu().numpy()
        assert np.abs(G - R).max() <= 1e-9 * np.abs(R).max()
    net, inp, _ = nets[0]
    s = solvers[0]
    T, B = 2, 2
    dem = np.stack([inp["demand"][:B] * f for f in (1.0, 1.05)])
    rh = np.nan_to_num(inp["res_head"][:B])
    th0 = np.broadcast_to(np.asarray(net.tank_h0), (B, len(net.tank_node))).copy()
    D = torch.tensor(dem, device=cuda).requires_grad_(True)
    out = eps_solve(s, D, torch.tensor(rh, device=cuda), torch.tensor(th0, device=cuda),
                    accuracy=1e-7)
    (out["head"] ** 2).sum().backward()
    eo = EpsOracle(net)
    runs = eo.run(dem, rh, th0, accuracy=1e-7)
    gH = [[2.0 * h for h in fr["head"]] for fr in runs]
    gQ = [[np.zeros(net.L) for _ in fr["head"]] for fr in runs]
    gE = [[np.zeros(net.N) for _ in fr["head"]] for fr in runs]
    gT = [[np.zeros(len(net.tank_node)) for _ in fr["head"]] for fr in runs]
    g_dem = eo.backward(runs, gH, gQ, gE, gT, P=T)[0]
    G = D.grad.cpu().numpy()
    assert np.abs(G - g_dem).max() <= 1e-7 * np.abs(g_dem).max()
