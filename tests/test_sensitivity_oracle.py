"""Sensitivity matrix pin: the oracle's per-sensor adjoints on its polished
state, times the H-W chain factor, against the reference's own
sensitivity_matrix (fixture tests/golden/sens_ref.npz, `make_golden.py sens`)."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

from golden.load import load  # noqa: E402
from oracle.gga import Model  # noqa: E402


def oracle_sensitivity(net, d, rh, sensors, wrt, accuracy=1e-10, model=None):
    """S[B*m, L]: one batched adjoint per sensor (unit right-hand side at that
    sensor in every frame), rows frame-major."""
    m = Model(net) if model is None else model
    out, st = m.implicit(d, rh, accuracy=accuracy)
    B, ms = d.shape[0], len(sensors)
    S = np.empty((B, ms, net.L))
    for c, i in enumerate(sensors):
        gH = np.zeros((B, net.N))
        gH[:, i] = 1.0
        S[:, c] = m.backward(st, gH, np.zeros((B, net.L)), np.zeros((B, net.N)))[3]
    S = S.reshape(B * ms, net.L)
    if wrt == "C":
        C = np.asarray(net.roughness)
        pipe = np.isin(np.asarray(net.link_type), (0, 1)) & (C > 0)
        chain = np.zeros(net.L)
        chain[pipe] = -1.852 * np.asarray(net.r_hw)[pipe] / C[pipe]
        S = S * chain[None, :]
    return S


def test_oracle_sensitivity_matches_reference():
    net, inp, ref = load("sens_ref")
    for wrt in ("C", "r"):
        S = oracle_sensitivity(net, inp["demand"], inp["res_head"], inp["sensors"], wrt)
        R = ref["S_" + wrt]
        assert S.shape == R.shape
        assert np.abs(S - R).max() <= 1e-6 * np.abs(R).max(), (wrt, np.abs(S - R).max())
