"""Flow control and pressure sustaining valve pins: the oracle's batched FCV
(valve-order fcvcoeff, fcvstatus at the link-status checks) and PSV
(psvcoeff, psvstatus, constraint rows at the upstream junction) against the
reference's EPANET replica with its status machine (fixtures
tests/golden/fcv_ref.npz and psv_ref.npz, `make_golden.py fcv` / `psv`):
iteration counts and statuses exact, heads, and the CPU implicit adjoint's
gradients with the final statuses frozen."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.gga import Model  # noqa: E402


def valve_loss_grads(m, net, inp, accuracy=1e-7):
    """Oracle implicit solve and the adjoint of L = sum h[sensors]^2 +
    sum q[loss links]^2 (the valve links the fixture names)."""
    d, rh = inp["demand"], inp["res_head"]
    out, st = m.implicit(d, rh, ke=inp["ke"], accuracy=accuracy)
    B = d.shape[0]
    fl = np.asarray(inp["loss_links"])
    H, q = out["head_ft"], out["flow_cfs"]
    gH = np.zeros((B, net.N))
    for b in range(B):
        np.add.at(gH[b], np.asarray(inp["sensors"]), 2.0 * H[b, inp["sensors"]])
    gQ = np.zeros((B, net.L))
    gQ[:, fl] = 2.0 * q[:, fl]
    return out, m.backward(st, gH, gQ, np.zeros((B, net.N)))


def test_oracle_fcv_forward_matches_reference():
    net, inp, ref = load("fcv_ref")
    out = Model(net).solve(inp["demand"], inp["res_head"], ke=inp["ke"], accuracy=1e-7,
                           status_machine=True)
    np.testing.assert_array_equal(out["iters"], ref["fwd_iters"].ravel())
    np.testing.assert_array_equal(out["status"], ref["fwd_status"])
    # raw GGA state (stops at relerr <= 1e-7): the two linear solvers' rounding
    # on a matrix with CBIG entries, as in the other raw-state comparisons
    assert np.abs(out["head_ft"] - ref["fwd_head"]).max() < 1e-4
    fl = np.flatnonzero(np.asarray(net.link_type) == 6)
    assert set(ref["fwd_status"][:, fl].ravel().tolist()) == {4, 6}   # ACTIVE and XFCV


def test_oracle_fcv_adjoint_matches_reference():
    net, inp, ref = load("fcv_ref")
    out, g = valve_loss_grads(Model(net), net, inp)
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-9
    fixed = np.asarray(net.node_type) != 0
    for gi, key, cols in ((g[0], "g_demand", slice(None)), (g[2], "g_ke", slice(None)),
                          (g[3], "g_rhw", slice(None)), (g[1], "g_res_head", fixed)):
        R = ref[key][:, cols]           # one reference call per scenario: per-scenario rows
        assert np.abs(gi[:, cols] - R).max() <= 1e-8 * np.abs(R).max(), (key, np.abs(gi[:, cols] - R).max())


def test_oracle_psv_matches_reference():
    """PSV pin (fixture tests/golden/psv_ref.npz): the ACTIVE PSV holds its
    upstream head; together with the network's ACTIVE PRV the adjoint has
    constraint rows of both orientations."""
    net, inp, ref = load("psv_ref")
    out = Model(net).solve(inp["demand"], inp["res_head"], ke=inp["ke"], accuracy=1e-7,
                           status_machine=True)
    np.testing.assert_array_equal(out["iters"], ref["fwd_iters"].ravel())
    np.testing.assert_array_equal(out["status"], ref["fwd_status"])
    assert np.abs(out["head_ft"] - ref["fwd_head"]).max() < 1e-4
    out, g = valve_loss_grads(Model(net), net, inp)
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-9
    fixed = np.asarray(net.node_type) != 0
    for gi, key, cols in ((g[0], "g_demand", slice(None)), (g[2], "g_ke", slice(None)),
                          (g[3], "g_rhw", slice(None)), (g[1], "g_res_head", fixed)):
        R = ref[key][:, cols]
        assert np.abs(gi[:, cols] - R).max() <= 1e-8 * np.abs(R).max(), (key, np.abs(gi[:, cols] - R).max())


def test_oracle_many_valves_match_reference():
    """Eight PRVs and two PSVs on one network (fixture
    tests/golden/valves_ref.npz): ten constraint rows, any valve count as in
    the reference's valve loop and Woodbury (dgga/solver.py:863,
    dgga/autodiff.py:965-1029)."""
    net, inp, ref = load("valves_ref")
    lt = np.asarray(net.link_type)
    assert (lt == 3).sum() == 8 and (lt == 4).sum() == 2
    out = Model(net).solve(inp["demand"], inp["res_head"], ke=inp["ke"], accuracy=1e-7,
                           status_machine=True)
    np.testing.assert_array_equal(out["iters"], ref["fwd_iters"].ravel())
    np.testing.assert_array_equal(out["status"], ref["fwd_status"])
    assert np.abs(out["head_ft"] - ref["fwd_head"]).max() < 1e-4
    v = np.flatnonzero((lt == 3) | (lt == 4))
    assert (ref["fwd_status"][:, v] == 4).sum() >= 35            # nearly every valve ACTIVE
    out, g = valve_loss_grads(Model(net), net, inp)
    assert np.abs(out["head_ft"] - ref["head"]).max() < 1e-9
    fixed = np.asarray(net.node_type) != 0
    for gi, key, cols in ((g[0], "g_demand", slice(None)), (g[2], "g_ke", slice(None)),
                          (g[3], "g_rhw", slice(None)), (g[1], "g_res_head", fixed)):
        R = ref[key][:, cols]
        assert np.abs(gi[:, cols] - R).max() <= 1e-8 * np.abs(R).max(), (key, np.abs(gi[:, cols] - R).max())
