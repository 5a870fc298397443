"""Flow control and pressure sustaining valves on the B200 route
(WDS_KIND_FCV, WDS_KIND_PSV): the batched GGA with FCVs in the valve pass and
fcvstatus, PSVs in the valve pass, psvstatus and the constraint rows at their
upstream junction, against the reference's EPANET replica with its status
machine (fixtures tests/golden/fcv_ref.npz, psv_ref.npz), its CPU implicit
adjoint, and the oracle on unseen scenarios."""
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

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["fcv_ref", "psv_ref", "valves_ref"])
def test_valve_forward_matches_reference(cuda, case):
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load(case)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    out = s.solve(torch.tensor(inp["demand"], device=cuda),
                  torch.tensor(inp["res_head"], device=cuda),
                  ke_int=torch.tensor(inp["ke"], device=cuda), accuracy=1e-7, status_machine=True)
    np.testing.assert_array_equal(out["iters"].cpu().numpy(), ref["fwd_iters"].ravel())
    np.testing.assert_array_equal(out["status"].cpu().numpy(), ref["fwd_status"])
    assert np.abs(out["head_ft"].cpu().numpy() - ref["fwd_head"]).max() < 1e-4


@pytest.mark.parametrize("case", ["fcv_ref", "psv_ref", "valves_ref"])
def test_valve_gradients_match_reference(cuda, case):
    from wdsgpu_b200.autodiff import implicit_solve
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load(case)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    B = inp["demand"].shape[0]
    D = torch.tensor(inp["demand"], device=cuda).requires_grad_(True)
    RH = torch.tensor(inp["res_head"], device=cuda).requires_grad_(True)
    KE = torch.tensor(np.tile(inp["ke"], (B, 1)), device=cuda).requires_grad_(True)
    R = torch.tensor(np.tile(np.asarray(net.r_hw), (B, 1)), device=cuda).requires_grad_(True)
    h, q, e = implicit_solve(s, D, RH, ke=KE, r_hw=R, accuracy=1e-7)
    fl = torch.as_tensor(np.asarray(inp["loss_links"]), device=cuda)
    sens = torch.as_tensor(np.asarray(inp["sensors"]), device=cuda)
    ((h[:, sens] ** 2).sum() + (q[:, fl] ** 2).sum()).backward()
    assert np.abs(h.detach().cpu().numpy() - ref["head"]).max() < 1e-9
    fixed = np.asarray(net.node_type) != 0
    for g, key, cols in ((D.grad, "g_demand", slice(None)), (KE.grad, "g_ke", slice(None)),
                         (R.grad, "g_rhw", slice(None)), (RH.grad, "g_res_head", fixed)):
        gi = g.cpu().numpy()[:, cols]
        Rf = ref[key][:, cols]
        assert np.abs(gi - Rf).max() <= 1e-8 * np.abs(Rf).max(), (key, np.abs(gi - Rf).max())


@pytest.mark.parametrize("which", ["fcv", "psv", "valves"])
def test_valve_unseen_scenarios_against_oracle(cuda, which):
    from wdsgpu_b200 import synth
    from wdsgpu_b200.autodiff import implicit_solve
    from wdsgpu_b200.solver import GGASolver
    net = {"fcv": synth.fcv_network, "psv": synth.psv_network,
           "valves": synth.many_valves_network}[which]()
    d, _ = synth.config2_scenarios(net, 12, seed=97, sigma=0.4)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    out = s.solve(torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda), accuracy=1e-7,
                  status_machine=True)
    m = Model(net)
    o = m.solve(d, rh, accuracy=1e-7, status_machine=True)
    np.testing.assert_array_equal(out["iters"].cpu().numpy(), o["iters"])
    np.testing.assert_array_equal(out["status"].cpu().numpy(), o["status"])
    h = implicit_solve(s, torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda),
                       accuracy=1e-7)[0]
    oi, _ = m.implicit(d, rh, accuracy=1e-7)
    assert np.abs(h.cpu().numpy() - oi["head_ft"]).max() < 1e-9 / 0.3048
