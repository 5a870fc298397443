"""Extended-period run on the B200 route, differentiable through time.

The reference has no batched or differentiable extended-period path; its
serial EPANET replica `EpsDriver` (dgga/eps.py) fixes the semantics of one
hydraulic step, which this module batches:

1. a steady solve with every tank as a fixed head (dgga/solver.py:223-230),
   warm started from the previous step's link and emitter flows (the q0 / e0
   keywords of GGASolver.solve, solver.py:2876-2887; EpsDriver.run keeps the
   flows from frame to frame, eps.py:366-373).  Here the solve is the
   implicit (polished) one, so each step ends at the Newton fixed point;
2. the net inflow of each tank: the flows of its links whose status is above
   CLOSED, + into the tank, - out of it (solver.py:2063-2073);
3. V += dt Q_net, then the one-second look-ahead clamp to [Vmin, Vmax]
   (EpsDriver._tanklevels, eps.py:278-291);
4. the new tank head, cylindrical: Hmin + (V - Vmin) / area
   (EpsDriver._tankgrade, eps.py:91-95).

Differences from EpsDriver, by design: the step is a fixed dt (EpsDriver
shortens a step when a tank would fill or empty inside it, or at a control
or pattern boundary), link statuses are re-derived by the status machine at
every step (EpsDriver carries them over), and controls and rules are not
applied.

Backward pass: adjoint through time.  Each step keeps a checkpoint (its tank
heads and warm start, a few numbers per scenario); walking the steps in
reverse, the step's polished forward is recomputed from the checkpoint, which
leaves that step's terminal factor in the plan, and one wds_adjoint launch
turns dL/d(heads, flows, emitter flows) of the step, plus the tank-volume
sensitivity carried from later steps, into dL/d(demand, reservoir heads, Ke,
r) of the step and dL/d(tank heads) carried to earlier steps.  A clamped
update carries nothing.  No factor of any step is stored.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .autodiff import _adjoint_guards, _clamp_grh, _clamp_rhs
from .solver import GGASolver, _check_emitter_cap, _not_pd_hint

__all__ = ["eps_solve", "EpsSM100", "tank_links"]

ST_CLOSED = 2


def tank_links(solver: GGASolver):
    """Links incident to tanks: (link index, tank index, sign) with sign +1
    when the link's end node n2 is the tank (its flow enters the tank) and -1
    when n1 is (solver.py:2063-2073)."""
    net = solver.net
    tn = np.asarray(net.tank_node if net.tank_node is not None else [], dtype=np.int64)
    pos = {int(n): j for j, n in enumerate(tn)}
    ks, js, sg = [], [], []
    for k in range(solver.L):
        a, b = int(net.link_n1[k]), int(net.link_n2[k])
        if a in pos:
            ks.append(k); js.append(pos[a]); sg.append(-1.0)
        if b in pos:
            ks.append(k); js.append(pos[b]); sg.append(1.0)
    return (np.asarray(ks, dtype=np.int64), np.asarray(js, dtype=np.int64),
            np.asarray(sg, dtype=np.float64))


class _Tanks:
    """Device-side tank tables of one solver."""

    def __init__(self, s: GGASolver):
        net = s.net
        dev = s.device
        f = lambda x: torch.as_tensor(np.asarray(x, dtype=np.float64), device=dev)
        self.node = torch.as_tensor(np.asarray(net.tank_node, dtype=np.int64), device=dev)
        self.nt = int(self.node.numel())
        self.area = f(net.tank_area)
        self.hmin = f(net.tank_hmin)
        self.vmin = f(net.tank_vmin)
        self.vmax = f(net.tank_vmax)
        ks, js, sg = tank_links(s)
        self.k = torch.as_tensor(ks, device=dev)
        self.j = torch.as_tensor(js, device=dev)
        self.sign = f(sg)

    def volume(self, h):
        """tankvolume, cylindrical (eps.py:86-89)."""
        return self.vmin + (h - self.hmin) * self.area

    def head(self, v):
        """tankgrade, cylindrical (eps.py:91-95)."""
        return self.hmin + (v - self.vmin) / self.area

    def inflow(self, flow, status):
        """Net inflow [B, nt] from the links above CLOSED."""
        B = flow.shape[0]
        q = flow.index_select(1, self.k) * (status.index_select(1, self.k) > ST_CLOSED)
        out = torch.zeros(B, self.nt, dtype=torch.float64, device=flow.device)
        return out.index_add_(1, self.j, q * self.sign)

    def step(self, v, qnet, dt):
        """tanklevels (eps.py:278-291): explicit Euler, then the one-second
        look-ahead clamp.  Returns (new volume, clamped mask)."""
        v = v + qnet * dt
        hi = v + qnet >= self.vmax
        lo = ~hi & (v - qnet <= self.vmin)
        v = torch.where(hi, self.vmax.expand_as(v), torch.where(lo, self.vmin.expand_as(v), v))
        return v, hi | lo


def _step_forward(s, d, rh, ke, r, B, max_iter, acc, polish, q0, e0):
    o = s.run(d, rh, ke, r, B, max_iter, acc, True, polish, q0=q0, e0=e0)
    info = o["info"]
    _check_emitter_cap(s, info)
    if bool((info != 0).any()):
        bad = torch.nonzero(info != 0).flatten().tolist()
        if bool((info & _lib.INFO_NOT_PD).any()):
            raise RuntimeError("eps: the node matrix of scenarios %s is not positive definite%s"
                               % (bad[:8], _not_pd_hint(s)))
        raise RuntimeError("eps: scenarios %s did not converge (relerr=%s > accuracy=%g)"
                           % (bad[:8], [float(o["relerr"][b]) for b in bad[:4]], acc))
    return o


class EpsSM100(torch.autograd.Function):
    """(demand[T,B,N], res_head[B,N], tank_h0[B,nt], ke[B or 1,N],
    r_hw[B or 1,L], solver, dt, accuracy, max_iter, polish_steps) ->
    (head[T,B,N], flow[T,B,L], emitter[T,B,N], tank_head[T+1,B,nt])."""

    @staticmethod
    def forward(ctx, demand, res_head, tank_h0, ke, r_hw, solver, dt, accuracy, max_iter,
                polish_steps):
        s = solver
        tk = _Tanks(s)
        T, B, N = demand.shape
        L = s.L
        dev = s.device
        d_all = demand.detach().contiguous()
        rh0 = res_head.detach().contiguous()
        ke_t = ke.detach().contiguous()
        r_t = r_hw.detach().contiguous()
        h = tank_h0.detach().clone()
        v = tk.volume(h)
        heads = torch.empty(T, B, N, dtype=torch.float64, device=dev)
        flows = torch.empty(T, B, L, dtype=torch.float64, device=dev)
        emits = torch.empty(T, B, N, dtype=torch.float64, device=dev)
        tank_heads = torch.empty(T + 1, B, tk.nt, dtype=torch.float64, device=dev)
        tank_heads[0] = h
        clamped = torch.empty(T, B, tk.nt, dtype=torch.bool, device=dev)
        opened = torch.empty(T, B, int(tk.k.numel()), dtype=torch.bool, device=dev)
        warm_q = torch.empty(T, B, L, dtype=torch.float64, device=dev)
        warm_e = torch.empty(T, B, N, dtype=torch.float64, device=dev)
        q0 = e0 = None
        for t in range(T):
            rh = rh0.clone()
            rh[:, tk.node] = h
            o = _step_forward(s, d_all[t], rh, ke_t, r_t, B, max_iter, accuracy,
                              polish_steps, q0, e0)
            _adjoint_guards(s, o["flow"], o["status"], allow_clamp=True)
            heads[t], flows[t], emits[t] = o["head"], o["flow"], o["emit"]
            # checkpoint of the step: its warm start (tank heads are tank_heads[t])
            if q0 is None:
                warm_q[t] = s._warm(s._tables["q_init"], B, L)
                warm_e[t] = torch.where(ke_t > 0, 1.0, 0.0).expand(B, N)
            else:
                warm_q[t], warm_e[t] = q0, e0
            opened[t] = o["status"].index_select(1, tk.k) > ST_CLOSED
            qnet = tk.inflow(o["flow"], o["status"])
            v, clamped[t] = tk.step(v, qnet, float(dt))
            h = tk.head(v)
            tank_heads[t + 1] = h
            q0, e0 = o["flow"].contiguous(), o["emit"].contiguous()
        ctx.save_for_backward(d_all, rh0, ke_t, r_t, tank_heads, clamped, opened,
                              warm_q, warm_e)
        ctx.solver, ctx.tk = s, tk
        ctx.args = (float(dt), float(accuracy), int(max_iter), int(polish_steps))
        ctx.kedim, ctx.rdim = ke.shape[0], r_hw.shape[0]
        return heads, flows, emits, tank_heads

    @staticmethod
    def backward(ctx, gH, gQ, gE, gT):
        if torch.is_grad_enabled():
            raise NotImplementedError("the extended-period adjoint is first order only")
        s, tk = ctx.solver, ctx.tk
        d_all, rh0, ke_t, r_t, tank_heads, clamped, opened, warm_q, warm_e = ctx.saved_tensors
        dt, acc, max_iter, polish = ctx.args
        T, B, N = d_all.shape
        L = s.L
        dev = s.device
        z = lambda *sh: torch.zeros(*sh, dtype=torch.float64, device=dev)
        gH = z(T, B, N) if gH is None else gH.to(torch.float64)
        gQ = z(T, B, L) if gQ is None else gQ.to(torch.float64)
        gE = z(T, B, N) if gE is None else gE.to(torch.float64)
        gT = z(T + 1, B, tk.nt) if gT is None else gT.to(torch.float64)
        g_dem = z(T, B, N)
        g_rh = z(B, N)
        g_ke = z(B, N)
        g_r = z(B, L)
        gV = gT[T] / tk.area                       # dL/dV_T
        for t in range(T - 1, -1, -1):
            free = ~clamped[t]
            gqnet = torch.where(free, gV * dt, 0.0)   # dL/dQnet_t
            gV = torch.where(free, gV, 0.0)           # dL/dV_t through V_{t+1}
            gq = gQ[t].clone()
            gq.index_add_(1, tk.k, gqnet.index_select(1, tk.j) * tk.sign * opened[t])
            rh = rh0.clone()
            rh[:, tk.node] = tank_heads[t]
            o = _step_forward(s, d_all[t], rh, ke_t, r_t, B, max_iter, acc, polish,
                              warm_q[t].contiguous(), warm_e[t].contiguous())
            gHt, gq, gEt = gH[t].contiguous(), gq.contiguous(), gE[t].contiguous()
            # constant-HP pumps on their clamp branch: Woodbury on the kept factor
            clamp = _adjoint_guards(s, o["flow"], o["status"], allow_clamp=True)
            fix = None
            if clamp is not None:
                gHt, fix = _clamp_rhs(s, o["plan"], B, clamp, gHt, gq, gEt,
                                      torch.cuda.current_stream(dev).cuda_stream)
            gd, grh, gke, gr = _adjoint_launch(s, o["plan"], B, gHt, gq, gEt)
            if fix is not None:
                _clamp_grh(fix, gq, gd, grh)
            g_dem[t] = gd
            g_rh += grh
            g_ke += gke
            g_r += gr
            gV = gV + (grh.index_select(1, tk.node) + gT[t]) / tk.area
        g_rh[:, tk.node] = 0.0                     # tank entries of res_head are not used
        g_h0 = gV * tk.area
        g_ke = g_ke.sum(0, keepdim=True) if ctx.kedim == 1 else g_ke
        g_r = g_r.sum(0, keepdim=True) if ctx.rdim == 1 else g_r
        return g_dem, g_rh, g_h0, g_ke, g_r, None, None, None, None, None


def _adjoint_launch(s, plan, B, gH, gQ, gE):
    import ctypes
    dev = s.device
    gd = torch.empty(B, s.N, dtype=torch.float64, device=dev)
    grh = torch.empty_like(gd)
    gke = torch.empty_like(gd)
    gr = torch.empty(B, s.L, dtype=torch.float64, device=dev)
    cur = torch.cuda.current_stream(dev)
    _lib.check(plan.lib.wds_adjoint(
        plan.handle, B, gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), gd.data_ptr(),
        grh.data_ptr(), gke.data_ptr(), gr.data_ptr(), ctypes.c_void_p(cur.cuda_stream)),
        "wds_adjoint")
    return gd, grh, gke, gr


def eps_solve(solver: GGASolver, demand, res_head=None, tank_h0=None, ke=None, r_hw=None,
              dt=3600.0, accuracy=1e-6, max_iter=200, polish_steps=3):
    """Batched extended-period run of T steps of dt seconds.

    demand [T,B,N] (cfs); res_head [B,N] or [N] fixed heads (ft; tank entries
    are ignored, default: the network's reservoir heads); tank_h0 [B,nt] or
    [nt] initial tank heads (default net.tank_h0); ke [N] or [B,N]; r_hw [L]
    or [B,L].  Returns dict(head [T,B,N], flow [T,B,L], emitter [T,B,N],
    tank_head [T+1,B,nt]), differentiable w.r.t. demand, res_head, tank_h0, ke
    and r_hw (1-D parameters receive the batch-summed gradient)."""
    s = solver
    dev = s.device
    if s.net.tank_node is None or len(s.net.tank_node) == 0:
        raise ValueError("eps_solve: the network has no tanks")
    t = lambda x: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    demand = t(demand)
    if demand.dim() != 3 or demand.shape[2] != s.N:
        raise ValueError("eps_solve: demand must be [T, B, N]")
    T, B, N = demand.shape
    if res_head is None:
        res_head = np.nan_to_num(s.net.fixed_head_ft_at(0))
    res_head = t(res_head)
    res_head = res_head.unsqueeze(0).expand(B, -1) if res_head.dim() == 1 else res_head
    tank_h0 = t(s.net.tank_h0 if tank_h0 is None else tank_h0)
    tank_h0 = tank_h0.unsqueeze(0).expand(B, -1) if tank_h0.dim() == 1 else tank_h0
    ke = t(s.node_ke_default if ke is None else ke)
    ke = ke.unsqueeze(0) if ke.dim() == 1 else ke
    r_hw = t(s.r_hw if r_hw is None else r_hw)
    r_hw = r_hw.unsqueeze(0) if r_hw.dim() == 1 else r_hw
    head, flow, emit, tank_head = EpsSM100.apply(demand, res_head, tank_h0, ke, r_hw, s,
                                                 float(dt), float(accuracy), int(max_iter),
                                                 int(polish_steps))
    return dict(head=head, flow=flow, emitter=emit, tank_head=tank_head)
