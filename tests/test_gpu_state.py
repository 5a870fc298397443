"""Terminal state kept per pending backward.

The reference keeps the factor of each implicit forward in its own autograd
context (dgga/autodiff.py:1203-1243), so `f(solve(d1)) + f(solve(d2))`
differentiates each call at its own state.  Here the factor lives in a plan's
workspace: a plan holding a pending backward's state is not given to later
forwards, and a state that was replaced anyway is refused by its generation."""
import numpy as np
import pytest
import torch

from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu


def _grad_alone(s, d, rh, sens, cuda):
    D = torch.tensor(d, device=cuda, requires_grad=True)
    h, _, _ = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-8)
    (h[:, sens] ** 2).sum().backward()
    return D.grad.detach().clone()


def test_two_forwards_then_two_backwards_match_single_calls(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    sens = torch.as_tensor(synth.sensor_nodes(net, 12), device=cuda)
    d1, rh = synth.config2_scenarios(net, 8, seed=501)
    d2, _ = synth.config2_scenarios(net, 8, seed=502)
    g1 = _grad_alone(s, d1, rh, sens, cuda)
    g2 = _grad_alone(s, d2, rh, sens, cuda)
    D1 = torch.tensor(d1, device=cuda, requires_grad=True)
    D2 = torch.tensor(d2, device=cuda, requires_grad=True)
    rht = torch.tensor(rh, device=cuda)
    h1, _, _ = implicit_solve(s, D1, rht, accuracy=1e-8)
    h2, _, _ = implicit_solve(s, D2, rht, accuracy=1e-8)      # a second plan holds this one
    assert sum(p.held for p in s._plans) == 2
    ((h1[:, sens] ** 2).sum() + (h2[:, sens] ** 2).sum()).backward()
    assert torch.equal(D1.grad, g1) and torch.equal(D2.grad, g2)
    assert not any(p.held for p in s._plans)                # claims end with the backward
    # separate backwards in the other order
    D1.grad = None
    D2.grad = None
    h1, _, _ = implicit_solve(s, D1, rht, accuracy=1e-8)
    h2, _, _ = implicit_solve(s, D2, rht, accuracy=1e-8)
    (h2[:, sens] ** 2).sum().backward()
    (h1[:, sens] ** 2).sum().backward()
    assert torch.equal(D1.grad, g1) and torch.equal(D2.grad, g2)


def test_replaced_state_is_refused_not_differentiated(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    sens = torch.as_tensor(synth.sensor_nodes(net, 6), device=cuda)
    d1, rh = synth.config2_scenarios(net, 4, seed=503)
    D = torch.tensor(d1, device=cuda, requires_grad=True)
    rht = torch.tensor(rh, device=cuda)
    h, _, _ = implicit_solve(s, D, rht, accuracy=1e-8)
    loss = (h[:, sens] ** 2).sum()
    loss.backward(retain_graph=True)                         # the claim ends here
    s.solve(torch.tensor(d1, device=cuda) * 1.1, rht, status_machine=True)  # reuses the plan
    with pytest.raises(RuntimeError, match="replaced by a later forward"):
        loss.backward()


def test_graph_freed_without_backward_releases_the_plan(cuda):
    net = synth.feature_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, _ = synth.config2_scenarios(net, 4, seed=504, sigma=0.3)
    rh = np.broadcast_to(net.fixed_head_ft_at(0), d.shape).copy()
    D = torch.tensor(d, device=cuda, requires_grad=True)
    out = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-8)
    assert any(p.held for p in s._plans)
    del out                                                  # the graph goes with its outputs
    assert not any(p.held for p in s._plans)
    with torch.no_grad():
        implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-8)
    assert not any(p.held for p in s._plans) and len(s._plans) == 1


def test_nan_reservoir_head_is_refused_and_the_solver_stays_usable(cuda):
    """A NaN head at a reservoir/tank node raises ValueError (as the reference
    does before its solve, dgga/solver.py:2892-2894); the forward kernel
    reports it per scenario and solves nothing for it, and the next call on
    the same solver is unaffected."""
    from wdsgpu_b200.autodiff import solve_unrolled
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    d, rh = synth.config2_scenarios(net, 4, seed=77)
    fixed = np.flatnonzero(np.asarray(net.node_type) != 0)
    bad = rh.copy()
    bad[2, fixed[0]] = np.nan
    ref = s.solve(d, rh, status_machine=True, accuracy=1e-8)
    with pytest.raises(ValueError, match="nan at a reservoir"):
        s.solve(d, bad, status_machine=True, accuracy=1e-8)
    with pytest.raises(ValueError, match="nan at a reservoir"):
        implicit_solve(s, torch.tensor(d, device=cuda, requires_grad=True),
                       torch.tensor(bad, device=cuda), accuracy=1e-8)
    s2 = GGASolver(synth.unrolled_network(), device=cuda, dense_status_machine=True)
    d2, rh2 = synth.config2_scenarios(s2.net, 2, seed=78)
    rh2 = np.nan_to_num(rh2)
    fx2 = np.flatnonzero(np.asarray(s2.net.node_type) != 0)
    rh2[1, fx2[0]] = np.nan
    with pytest.raises(ValueError, match="nan at a reservoir"):
        solve_unrolled(s2, torch.tensor(d2, device=cuda), torch.tensor(rh2, device=cuda), K=4)
    again = s.solve(d, rh, status_machine=True, accuracy=1e-8)
    assert torch.equal(again["head_ft"], ref["head_ft"])
