"""Sensor sensitivity matrix on the kept factor: S = dp_sensor / dC (or / dr).

Mirrors dgga/sensitivity.py:59-145 (`sensitivity_matrix`).  The reference
factorises the Jacobian once per frame and solves m sensor columns with it;
here one implicit forward keeps each scenario's terminal factor on the GPU and
`wds_adjoint_rhs` runs the m adjoints of every frame on it (row v = frame
v // m, sensor v % m), in launches of up to the plan's capacity.  No new
factorisation.  dp_i/dr_k = dH_i/dr_k (p = H - El); the C chain factor is
dr/dC = -Hexp r / C on H-W pipes and 0 elsewhere (dgga/calib.py dr_dC).
"""
from __future__ import annotations

import ctypes
from time import perf_counter

import numpy as np
import torch

from . import _lib
from .solver import GGASolver, _check_info_flags, _not_pd_hint

__all__ = ["sensitivity_matrix", "dr_dC_chain"]

_PIPE_KINDS = (0, 1)      # CVPIPE, PIPE


def dr_dC_chain(solver: GGASolver, r_hw=None):
    """dr/dC = -Hexp r / C on H-W pipes with C > 0, 0 elsewhere ([L] numpy)."""
    net = solver.net
    r = np.asarray(solver.r_hw.cpu().numpy() if r_hw is None else
                   (r_hw.detach().cpu().numpy() if isinstance(r_hw, torch.Tensor) else r_hw),
                   dtype=np.float64)
    C = np.asarray(net.roughness, dtype=np.float64)
    is_pipe = np.isin(np.asarray(net.link_type), _PIPE_KINDS) & (C > 0.0)
    out = np.zeros(solver.L, dtype=np.float64)
    out[is_pipe] = -solver.hexp * r[is_pipe] / C[is_pipe]
    return out


def sensitivity_matrix(solver, demand, res_head, r_hw, sensor_nodes, wrt="C", frames=None,
                       ke=None, accuracy=1e-12, max_iter=200, polish_steps=3, speed=None,
                       status=None, pump_h0=None, pump_r=None, return_info=False):
    """S[T*m, L] = dp_sensor/dtheta, theta = C (roughness) or r (r_hw), rows
    frame-major ([frame 0's m rows; frame 1's m rows; ...]), as the reference.
    speed / pump_h0 / pump_r ([L] or [T, L]) set the frames' pump parameters
    as in implicit_solve."""
    s = solver
    if wrt not in ("C", "r"):
        raise ValueError("wrt must be 'C' or 'r'")
    if status is not None:
        raise NotImplementedError(
            "status is not taken by the B200 route (the batched status machine decides "
            "each frame's status)")
    sensors = np.asarray(sensor_nodes, dtype=np.int64).ravel()
    nt = np.asarray(s.net.node_type)
    bad = sensors[nt[sensors] != 0]
    if bad.size:
        raise ValueError("sensor nodes %s are not junctions (a fixed head is an input, "
                         "dp/dC = 0 there)" % bad.tolist())
    m = sensors.size
    t0 = perf_counter()
    ke = s.node_ke_default if ke is None else ke
    r_hw = s.r_hw if r_hw is None else r_hw
    d, rh, ke_t, r_t, B, _ = s._inputs(demand, res_head, ke, r_hw)
    pumps = s.pump_rows(B, speed, pump_h0, pump_r)
    o = s.run(d, rh, ke_t.contiguous(), r_t.contiguous(), B, int(max_iter), float(accuracy),
              True, int(polish_steps), pumps=pumps)
    info_v = o["info"]
    _check_info_flags(s, info_v)
    if bool((info_v != 0).any()):
        badb = torch.nonzero(info_v != 0).flatten().tolist()
        if bool((info_v & _lib.INFO_NOT_PD).any()):
            raise RuntimeError("sensitivity_matrix: the node matrix of scenarios %s is not "
                               "positive definite%s" % (badb[:8], _not_pd_hint(s)))
        raise RuntimeError("sensitivity_matrix: scenarios %s did not converge" % badb[:8])
    torch.cuda.synchronize(s.device)
    t_forward = perf_counter() - t0
    plan = o["plan"]
    dev = s.device
    fr = list(range(B)) if frames is None else [int(b) for b in frames]
    rows = B * m
    cap = plan.max_batch
    S = np.empty((rows, s.L))
    sens_t = torch.as_tensor(sensors, device=dev)
    cur = torch.cuda.current_stream(dev)
    t1 = perf_counter()
    for v0 in range(0, rows, cap):
        nb = min(cap, rows - v0)
        gH = torch.zeros(nb, s.N, dtype=torch.float64, device=dev)
        v = torch.arange(v0, v0 + nb, device=dev)
        gH[torch.arange(nb, device=dev), sens_t[v % m]] = 1.0
        gQ = torch.zeros(nb, s.L, dtype=torch.float64, device=dev)
        gE = torch.zeros(nb, s.N, dtype=torch.float64, device=dev)
        gd = torch.empty(nb, s.N, dtype=torch.float64, device=dev)
        grh, gke = torch.empty_like(gd), torch.empty_like(gd)
        gr = torch.empty(nb, s.L, dtype=torch.float64, device=dev)
        _lib.check(plan.lib.wds_adjoint_rhs(
            plan.handle, nb, m, v0, gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), gd.data_ptr(),
            grh.data_ptr(), gke.data_ptr(), gr.data_ptr(), ctypes.c_void_p(cur.cuda_stream)),
            "wds_adjoint_rhs")
        S[v0:v0 + nb] = gr.cpu().numpy()
    t_adj = perf_counter() - t1
    if wrt == "C":
        S = S * dr_dC_chain(s, r_hw if r_hw is not None else None)[None, :]
    S = S.reshape(B, m, s.L)[fr].reshape(len(fr) * m, s.L)
    if return_info:
        return S, dict(frames=fr, sensors=sensors, n_factorizations=0, n_rhs=len(fr) * m,
                       t_forward=t_forward, t_adjoint=t_adj)
    return S
