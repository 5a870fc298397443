"""Sensor sensitivity matrix on the kept factor (wds_adjoint_rhs): against the
reference's own sensitivity_matrix (fixture tests/golden/sens_ref.npz), with
no new factorisation; also in launches smaller than the row count."""
import os
import sys

import numpy as np
import pytest
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402

pytestmark = pytest.mark.gpu


def test_sensitivity_matrix_matches_reference(cuda):
    from wdsgpu_b200.sensitivity import sensitivity_matrix
    from wdsgpu_b200.solver import GGASolver
    net, inp, ref = load("sens_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    for wrt in ("C", "r"):
        S, info = sensitivity_matrix(s, inp["demand"], inp["res_head"], None, inp["sensors"],
                                     wrt=wrt, accuracy=1e-10, return_info=True)
        R = ref["S_" + wrt]
        assert S.shape == R.shape and info["n_factorizations"] == 0
        assert np.abs(S - R).max() <= 1e-6 * np.abs(R).max(), (wrt, np.abs(S - R).max())
    # frames subset, rows in frame-major order
    S1 = sensitivity_matrix(s, inp["demand"], inp["res_head"], None, inp["sensors"], wrt="r",
                            frames=[1], accuracy=1e-10)
    m = len(inp["sensors"])
    assert np.abs(S1 - ref["S_r"][m:]).max() <= 1e-6 * np.abs(ref["S_r"]).max()


def test_sensitivity_rows_in_several_launches(cuda):
    """More rows (frames x sensors) than the plan holds: the rows go in
    several launches and agree with the oracle's per-sensor adjoints."""
    from wdsgpu_b200 import synth
    from wdsgpu_b200.sensitivity import sensitivity_matrix
    from wdsgpu_b200.solver import GGASolver
    from test_sensitivity_oracle import oracle_sensitivity
    net = synth.feature_network()
    d, _ = synth.config2_scenarios(net, 3, seed=71, sigma=0.2)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    sens = synth.sensor_nodes(net, 9, seed=2)
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    # 27 rows, the plan holds 4; accuracy 1e-7 as the feature golden cases
    # (its GGA relerr stalls above 1e-10)
    S = sensitivity_matrix(s, d, rh, None, sens, wrt="r", accuracy=1e-7)
    R = oracle_sensitivity(net, d, rh, sens, "r", accuracy=1e-7)
    assert np.abs(S - R).max() <= 1e-6 * np.abs(R).max()


def test_sensitivity_at_call_pump_speeds(cuda):
    """speed / pump_h0 / pump_r of the call set the frames' pumps (the
    reference's sensitivity_matrix takes them likewise)."""
    from wdsgpu_b200.sensitivity import sensitivity_matrix
    from wdsgpu_b200.solver import GGASolver
    from test_sensitivity_oracle import oracle_sensitivity   # puts the repo root on sys.path
    from oracle.gga import Model
    net, inp, _ = load("pump_ref")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    S = sensitivity_matrix(s, inp["demand"], inp["res_head"], None, inp["sensors"], wrt="r",
                           accuracy=1e-7, speed=inp["speed"], pump_h0=inp["pump_h0"],
                           pump_r=inp["pump_r"])
    m = Model(net).with_pumps(inp["speed"], inp["pump_h0"], inp["pump_r"])
    R = oracle_sensitivity(net, inp["demand"], inp["res_head"], inp["sensors"], "r",
                           accuracy=1e-7, model=m)
    assert np.abs(S - R).max() <= 1e-8 * np.abs(R).max()
    S0 = sensitivity_matrix(s, inp["demand"], inp["res_head"], None, inp["sensors"], wrt="r",
                            accuracy=1e-7)
    assert np.abs(S - S0).max() > 1e-6 * np.abs(R).max()     # the speeds matter
