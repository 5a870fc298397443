"""Parity of the sm_100a route against the reference (golden fixtures) and the
CPU oracle, plus the reference's own invariants: batched = single bitwise,
adjoint = central difference, torch.autograd.gradcheck, refusal instead of
fallback.  Every call goes through the C ABI (libwds_b200.so)."""
import numpy as np
import pytest
import torch

from oracle.gga import Model
from tests.golden.load import CASES, load
from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu

FWD_HEAD_ATOL_FT = 1e-4            # raw GGA state (stops at relerr <= accuracy)
POLISHED_HEAD_ATOL_FT = 1e-9 / 0.3048
POLISHED_FLOW_ATOL = 1e-9          # cfs
GRAD_RTOL = 1e-6


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _np(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module", params=CASES)
def golden(request, cuda):
    net, inp, ref = load(request.param)
    sm = bool(inp["status_machine"])
    s = GGASolver(net, device=cuda, dense_status_machine=sm)
    return request.param, net, inp, ref, s


def test_forward_matches_reference_golden(golden, cuda):
    tag, net, inp, ref, s = golden
    sm = bool(inp["status_machine"])
    out = s.solve(torch.tensor(inp["demand"], device=cuda),
                  torch.tensor(inp["res_head"], device=cuda),
                  ke_int=torch.tensor(inp["ke"], device=cuda),
                  accuracy=float(inp["accuracy"]), status_machine=sm)
    np.testing.assert_array_equal(_np(out["iters"]), ref["fwd_iters"])
    np.testing.assert_array_equal(_np(out["converged"]), ref["fwd_converged"])
    if sm:
        np.testing.assert_array_equal(_np(out["status"]), ref["fwd_status"])
    assert np.abs(_np(out["head_ft"]) - ref["fwd_head"]).max() < FWD_HEAD_ATOL_FT
    assert np.abs(_np(out["emitter_cfs"]) - ref["fwd_emitter"]).max() < 1e-5


def test_implicit_state_and_gradients_match_reference_golden(golden, cuda):
    tag, net, inp, ref, s = golden
    sm = bool(inp["status_machine"])
    D = torch.tensor(inp["demand"], device=cuda, requires_grad=True)
    KE = torch.tensor(inp["ke"][0], device=cuda, requires_grad=True)
    R = torch.tensor(np.asarray(net.r_hw), device=cuda, requires_grad=True)
    h, q, e = implicit_solve(s, D, torch.tensor(inp["res_head"], device=cuda), ke=KE, r_hw=R,
                             accuracy=float(inp["accuracy"]), polish_steps=3,
                             status_machine=sm)
    (h[:, inp["sensors"]] ** 2).sum().backward()
    assert np.abs(_np(h) - ref["imp_head"]).max() < POLISHED_HEAD_ATOL_FT
    assert np.abs(_np(q) - ref["imp_flow"]).max() < POLISHED_FLOW_ATOL
    assert np.abs(_np(e) - ref["imp_emitter"]).max() < POLISHED_FLOW_ATOL
    assert _rel(_np(D.grad), ref["grad_demand"]) < GRAD_RTOL
    assert _rel(_np(R.grad), ref["grad_r"]) < GRAD_RTOL
    if np.abs(ref["grad_ke"]).max() > 0:
        assert _rel(_np(KE.grad), ref["grad_ke"]) < GRAD_RTOL


def test_config2_against_oracle_fresh_seed(cuda):
    """Unseen scenarios of the 782-junction network: polished heads within
    1e-9 m and demand/roughness/emitter gradients within 1e-6 of the oracle."""
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 6, seed=123)
    sens = synth.sensor_nodes(net, 30)
    m = Model(net)
    out, st = m.implicit(d, rh, accuracy=1e-6, polish_steps=3, status_machine=True)
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd, grh, gke, gr = m.backward(st, gH, np.zeros_like(out["flow_cfs"]),
                                  np.zeros_like(out["emitter_cfs"]))
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    D = torch.tensor(d, device=cuda, requires_grad=True)
    KE = torch.tensor(net.node_ke, device=cuda, requires_grad=True)
    R = torch.tensor(net.r_hw, device=cuda, requires_grad=True)
    RH = torch.tensor(rh, device=cuda, requires_grad=True)
    h, q, e = implicit_solve(s, D, RH, ke=KE, r_hw=R, accuracy=1e-6, status_machine=True)
    (h[:, sens] ** 2).sum().backward()
    assert np.abs(_np(h) - out["head_ft"]).max() < POLISHED_HEAD_ATOL_FT
    assert _rel(_np(D.grad), gd) < GRAD_RTOL
    assert _rel(_np(R.grad), gr.sum(0)) < GRAD_RTOL
    assert _rel(_np(KE.grad), gke.sum(0)) < GRAD_RTOL
    assert _rel(_np(RH.grad), grh) < GRAD_RTOL


@pytest.mark.parametrize("accuracy", [1e-2, 1e-4])
def test_polish_factor_reuse_at_loose_accuracy(cuda, accuracy):
    """A loose GGA accuracy moves the Jacobian between polish steps, so the
    polish re-factors where needed and reuses a factor only within its
    per-entry bound: polished heads, flows and gradients still agree with
    the oracle's full Newton polish (which re-factors at every step)."""
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 6, seed=321)
    sens = synth.sensor_nodes(net, 30)
    m = Model(net)
    out, st = m.implicit(d, rh, accuracy=accuracy, polish_steps=3, status_machine=True)
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd = m.backward(st, gH, np.zeros_like(out["flow_cfs"]), np.zeros_like(out["emitter_cfs"]))[0]
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    D = torch.tensor(d, device=cuda, requires_grad=True)
    h, q, e = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=accuracy,
                             status_machine=True)
    (h[:, sens] ** 2).sum().backward()
    assert np.abs(_np(h) - out["head_ft"]).max() < POLISHED_HEAD_ATOL_FT
    assert _rel(_np(D.grad), gd) < GRAD_RTOL
    # three polish steps from a loose state leave both codes about 1e-10 of
    # the flows away from the root, from raw states that differ by rounding
    assert np.abs(_np(q) - out["flow_cfs"]).max() < 1e-9 * np.abs(out["flow_cfs"]).max()
    assert np.abs(_np(e) - out["emitter_cfs"]).max() < 1e-9 * np.abs(out["flow_cfs"]).max()


def test_batched_equals_single_bitwise(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = synth.config2_scenarios(net, 4, seed=5)
    D, RH = torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda)
    hb = implicit_solve(s, D, RH, accuracy=1e-6)[0]
    fb = s.solve(D, RH, accuracy=1e-6, status_machine=True)
    for b in range(4):
        h1 = implicit_solve(s, D[b], RH[b], accuracy=1e-6)[0]
        assert torch.equal(h1, hb[b])
        f1 = s.solve(D[b], RH[b], accuracy=1e-6, status_machine=True)
        assert int(f1["iters"]) == int(fb["iters"][b])
        assert torch.equal(f1["head_ft"], fb["head_ft"][b])


def test_repeat_calls_are_deterministic(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = synth.config2_scenarios(net, 64, seed=9)
    D, RH = torch.tensor(d, device=cuda, requires_grad=True), torch.tensor(rh, device=cuda)
    outs, grads = [], []
    for _ in range(2):
        D.grad = None
        h = implicit_solve(s, D, RH, accuracy=1e-6)[0]
        h.sum().backward()
        outs.append(h.detach().clone())
        grads.append(D.grad.clone())
    assert torch.equal(outs[0], outs[1])
    assert torch.equal(grads[0], grads[1])


def test_adjoint_matches_central_difference(cuda):
    """The reference gate (tests/test_smoke.py:81-98): rel < 1e-6, h = 1e-3 d."""
    for net in (synth.config1_network(), synth.config2_network()):
        sm = bool((np.asarray(net.link_type) == 3).any())
        s = GGASolver(net, device=cuda, dense_status_machine=sm)
        d = torch.tensor(net.demand_cfs_at(0), device=cuda)
        rh = torch.tensor(net.reservoir_head_ft_at(0), device=cuda)
        junc = np.flatnonzero(net.demand_cfs_at(0) > 0)
        i_theta, i_probe = int(junc[0]), int(junc[-1])
        dd = d.clone().requires_grad_(True)
        acc = 1e-9 if not sm else 1e-6
        head = implicit_solve(s, dd, rh, accuracy=acc, status_machine=sm)[0]
        head[i_probe].backward()
        g = float(dd.grad[i_theta])
        h = 1e-3 * float(d[i_theta])

        def head_at(delta):
            dp = d.clone()
            dp[i_theta] += delta
            return float(implicit_solve(s, dp, rh, accuracy=acc, status_machine=sm)[0][i_probe])

        fd = (head_at(h) - head_at(-h)) / (2 * h)
        assert abs(g - fd) / abs(fd) < 1e-6


def test_gradcheck_small_network(cuda):
    net = synth.config1_network()
    s = GGASolver(net, device=cuda)
    d = torch.tensor(net.demand_cfs_at(0), device=cuda).unsqueeze(0)
    rh = torch.tensor(net.reservoir_head_ft_at(0), device=cuda).unsqueeze(0)
    sens = synth.sensor_nodes(net, 5)
    d = d.requires_grad_(True)

    def f(dd):
        return implicit_solve(s, dd, rh, accuracy=1e-9)[0][:, sens]

    assert torch.autograd.gradcheck(f, (d,), eps=1e-6, atol=1e-5, rtol=1e-3)


def test_refuses_instead_of_falling_back(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d = torch.tensor(net.demand_cfs_at(0), device=cuda)
    rh = torch.tensor(net.reservoir_head_ft_at(0), device=cuda)
    out = s.solve(d, rh, max_iter=2, accuracy=1e-9, status_machine=True)
    assert not bool(out["converged"])
    assert int(out["iters"]) == 3                    # maxtrials + 1
    with pytest.raises(RuntimeError):
        implicit_solve(s, d, rh, max_iter=2, accuracy=1e-9)
    dd = d.clone().requires_grad_(True)
    h = implicit_solve(s, dd, rh, accuracy=1e-6)[0]
    with pytest.raises(NotImplementedError):
        torch.autograd.grad(h.sum(), dd, create_graph=True)


def test_full_batch_config2_properties(cuda):
    """B=1024 on the 782-junction network: every scenario converges, the
    polished state satisfies the nonlinear equations, and a sample of eight
    scenarios agrees with the oracle to 1e-9 m and 1e-6 on gradients."""
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = synth.config2_scenarios(net, 1024, seed=7)
    D = torch.tensor(d, device=cuda, requires_grad=True)
    h, q, e = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-6)
    sens = synth.sensor_nodes(net, 30)
    (h[:, sens] ** 2).sum().backward()
    assert torch.isfinite(D.grad).all()
    # one scenario from every (round, group slot) pair of the persistent CTAs
    # (148 CTAs x 3 groups on a B200: scenario (round * 3 + group) * 148 + cta),
    # plus the first and the last
    pick = np.array([0] + [k * 148 + (37 * k) % 136 for k in range(1, 7)] + [1023])
    m = Model(net)
    out, st = m.implicit(d[pick], rh[pick], accuracy=1e-6)
    assert np.abs(_np(h)[pick] - out["head_ft"]).max() < POLISHED_HEAD_ATOL_FT
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd = m.backward(st, gH, np.zeros_like(out["flow_cfs"]), np.zeros_like(out["emitter_cfs"]))[0]
    assert _rel(_np(D.grad)[pick], gd) < GRAD_RTOL
    # the persistent CTAs take scenario b = (round * groups + group) * CTAs + cta
    # (148 CTAs x 3 groups on a B200): scenarios from the second and third
    # group slot and from the later rounds, solved alone (round 0, group 0),
    # give the same bits, heads and gradients
    hd, gdd = _np(h), _np(D.grad)
    for b in (200, 400, 600, 887, 1000):
        Db = torch.tensor(d[b], device=cuda, requires_grad=True)
        hb = implicit_solve(s, Db, torch.tensor(rh[b], device=cuda), accuracy=1e-6)[0]
        (hb[sens] ** 2).sum().backward()
        assert np.array_equal(_np(hb), hd[b]), b
        assert np.array_equal(_np(Db.grad), gdd[b]), b
    # mass balance at every junction of every scenario
    qn = _np(q)
    n1, n2 = np.asarray(net.link_n1), np.asarray(net.link_n2)
    junc = np.flatnonzero(np.asarray(net.node_type) == 0)
    bal = np.zeros((1024, net.N))
    np.add.at(bal.T, n2, qn.T)
    np.add.at(bal.T, n1, -qn.T)
    bal -= d + _np(e)
    assert np.abs(bal[:, junc]).max() < 1e-9


def test_refine_band_keeps_iterations_and_statuses(cuda):
    """The default schedule (GGA solves refined once, and only once relerr <
    1e-5, at accuracy >= 1e-8) against the reference's schedule (every GGA
    solve refined twice, refine_band = 0) on 256 unseen config-2 scenarios:
    identical iteration counts and statuses, polished state within 1e-9 m."""
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    assert s.refine_band(1e-6) == 1e-5 and s.refine_band(1e-12) == 0.0
    assert s.refine_steps(1e-6) == 1 and s.refine_steps(1e-12) == 2
    d, rh = synth.config2_scenarios(net, 256, seed=404)
    d = torch.tensor(d, device=cuda)
    rh = torch.tensor(rh, device=cuda)
    ke = s.node_ke_default.unsqueeze(0).contiguous()
    r = s.r_hw.unsqueeze(0).contiguous()
    a = s.run(d, rh, ke, r, 256, 200, 1e-6, True, 3)
    b = s.run(d, rh, ke, r, 256, 200, 1e-6, True, 3, refine=2, refine_band=0.0)
    assert int(a["info"].abs().sum()) == 0 and int(b["info"].abs().sum()) == 0
    assert torch.equal(a["iters"], b["iters"])
    assert torch.equal(a["status"], b["status"])
    assert float((a["head"] - b["head"]).abs().max()) <= POLISHED_HEAD_ATOL_FT
    assert float((a["flow"] - b["flow"]).abs().max()) <= POLISHED_FLOW_ATOL
