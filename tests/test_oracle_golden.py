"""The CPU oracle against golden vectors produced by the reference itself
(tests/golden/make_golden.py).  This pins the oracle before it is used to
check the CUDA path."""
import numpy as np
import pytest

from oracle.gga import Model
from tests.golden.load import CASES, load

# raw GGA heads stop at relerr <= accuracy on matrices with condition ~1e10;
# two correct linear solvers differ there by ~1e-6..1e-5 ft
FWD_HEAD_ATOL_FT = 1e-4
# the polished fixed point: 1e-9 m expressed in ft
POLISHED_HEAD_ATOL_FT = 1e-9 / 0.3048
GRAD_RTOL = 1e-6


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.fixture(scope="module", params=CASES)
def case(request):
    net, inp, ref = load(request.param)
    return request.param, net, inp, ref, Model(net)


def test_forward_matches_reference(case):
    tag, net, inp, ref, m = case
    sm = bool(inp["status_machine"])
    out = m.solve(inp["demand"], inp["res_head"], ke=inp["ke"],
                  accuracy=float(inp["accuracy"]), status_machine=sm)
    np.testing.assert_array_equal(out["iters"], ref["fwd_iters"])
    np.testing.assert_array_equal(out["converged"], ref["fwd_converged"])
    if sm:
        np.testing.assert_array_equal(out["status"], ref["fwd_status"])
    assert np.abs(out["head_ft"] - ref["fwd_head"]).max() < FWD_HEAD_ATOL_FT


def test_polished_state_and_gradients_match_reference(case):
    tag, net, inp, ref, m = case
    sm = bool(inp["status_machine"])
    out, st = m.implicit(inp["demand"], inp["res_head"], ke=inp["ke"][0],
                         accuracy=float(inp["accuracy"]), polish_steps=3,
                         status_machine=sm)
    assert np.abs(out["head_ft"] - ref["imp_head"]).max() < POLISHED_HEAD_ATOL_FT
    assert np.abs(out["flow_cfs"] - ref["imp_flow"]).max() < 1e-9
    sens = inp["sensors"]
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd, grh, gke, gr = m.backward(st, gH, np.zeros_like(out["flow_cfs"]),
                                  np.zeros_like(out["emitter_cfs"]))
    assert _rel(gd, ref["grad_demand"]) < GRAD_RTOL
    assert _rel(gr.sum(0), ref["grad_r"]) < GRAD_RTOL
    if np.abs(ref["grad_ke"]).max() > 0:
        assert _rel(gke.sum(0), ref["grad_ke"]) < GRAD_RTOL


def test_gpu_route_algorithm_agrees_with_epanet_replica_adjoint():
    """cfg1 also carries the reference's EPANET-replica + splu adjoint; the
    oracle's reduced adjoint must agree with it (two independent methods)."""
    net, inp, ref = load("cfg1")
    m = Model(net)
    out, st = m.implicit(inp["demand"], inp["res_head"], ke=inp["ke"][0],
                         accuracy=float(inp["accuracy"]))
    assert np.abs(out["head_ft"] - ref["cpu_head"]).max() < 1e-8
    sens = inp["sensors"]
    gH = np.zeros_like(out["head_ft"])
    gH[:, sens] = 2.0 * out["head_ft"][:, sens]
    gd, grh, gke, gr = m.backward(st, gH, np.zeros_like(out["flow_cfs"]),
                                  np.zeros_like(out["emitter_cfs"]))
    assert _rel(gd, ref["cpu_grad_demand"]) < 1e-6
    assert _rel(gr.sum(0), ref["cpu_grad_r"]) < 1e-6


def test_oracle_adjoint_matches_central_difference():
    """dL/d(demand) of the oracle against a central difference of the
    polished solve (the reference's own gate: rel < 1e-6, h = 1e-3 d)."""
    net, inp, ref = load("cfg1")
    m = Model(net)
    d = inp["demand"][:1].copy()
    rh = inp["res_head"][:1]
    sens = int(inp["sensors"][0])
    out, st = m.implicit(d, rh, accuracy=1e-12)
    gH = np.zeros_like(out["head_ft"])
    gH[0, sens] = 1.0
    gd, _, _, _ = m.backward(st, gH, np.zeros_like(out["flow_cfs"]),
                             np.zeros_like(out["emitter_cfs"]))
    j = int(np.flatnonzero(d[0] > 0)[0])
    h = 1e-3 * d[0, j]

    def head(delta):
        dp = d.copy()
        dp[0, j] += delta
        return m.implicit(dp, rh, accuracy=1e-12)[0]["head_ft"][0, sens]

    fd = (head(h) - head(-h)) / (2 * h)
    assert abs(gd[0, j] - fd) / abs(fd) < 1e-6
