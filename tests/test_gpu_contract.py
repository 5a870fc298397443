"""The rest of GGASolver.solve's result contract against the reference
(fixture tests/golden/contract_ref.npz, `make_golden.py contract`):

* `diag_ratio`, the condition proxy max |A_jj| / min |A_jj| of the last GGA
  iteration's node matrix on networks with PRVs (dgga/solver.py:3026-3032,
  3205-3207).  The raw GGA states of the two linear solvers differ by their
  rounding (raw heads within 1e-4 ft), so the ratio is compared at 1e-5
  relative;
* the status-machine schedule of record_schedule=True (:2740-2745,
  3136-3160): every valve-pass and link-status entry, its iteration, its
  per-scenario flags and its change bitmap, exactly."""
import os

import numpy as np
import pytest
import torch

from tests.golden.load import load
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ("cfg2", "feat_mid", "feat_low", "cfg3_tcv")


@pytest.fixture(scope="module")
def contract():
    return np.load(os.path.join(HERE, "golden", "contract_ref.npz"))


@pytest.mark.parametrize("tag", TAGS)
def test_diag_ratio_and_schedule_match_reference(cuda, contract, tag):
    net, inp, ref = load(tag)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    out = s.solve(torch.tensor(inp["demand"], device=cuda),
                  torch.tensor(inp["res_head"], device=cuda),
                  ke_int=torch.tensor(inp["ke"], device=cuda),
                  accuracy=float(inp["accuracy"]), status_machine=True, record_schedule=True)
    np.testing.assert_array_equal(out["iters"].cpu().numpy(), ref["fwd_iters"])
    key = tag + "__diag_ratio"
    if key in contract.files:
        dr = out["diag_ratio"].cpu().numpy()
        np.testing.assert_allclose(dr, contract[key], rtol=1e-5)
    else:
        assert "diag_ratio" not in out
    sch = out["schedule"]
    its = contract[tag + "__sched_it"]
    assert [e["it"] for e in sch] == its.tolist()
    for i, e in enumerate(sch):
        valve = bool(contract[tag + "__sched_valve"][i])
        assert (e.get("kind") == "valve") == valve, i
        if valve:
            np.testing.assert_array_equal(e["act"], contract[tag + "__sched_a"][i])
        else:
            np.testing.assert_array_equal(e["conv"], contract[tag + "__sched_a"][i])
            np.testing.assert_array_equal(e["per"], contract[tag + "__sched_b"][i])
        np.testing.assert_array_equal(e["chg"], contract[tag + "__sched_chg"][i])


def test_record_schedule_needs_the_status_machine(cuda):
    net, inp, _ = load("cfg1")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    with pytest.raises(ValueError, match="record_schedule"):
        s.solve(inp["demand"], inp["res_head"], record_schedule=True)
