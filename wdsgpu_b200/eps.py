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

As in EpsDriver, frames follow the reference's clock: after the frame at
Htime the time step is min(Hstep, time to the next pattern boundary, to the
next report time, to the first tank filling or emptying, ROUND of volume
over net inflow; EpsDriver._timestep and _tanktimestep, eps.py:262-276,
211-229), so every scenario has its own frame times; link flows, emitter
flows and link statuses carry from frame to frame (run_gga(q0, e0,
status0), eps.py:366-373).  The frames of one launch are the frames of all
scenarios at the same index; a scenario that reached the end early has
padding frames (valid False, zero outputs, no gradient).  Controls and rules
(EpsDriver._controls, the rule engine) are not applied.

Backward pass: adjoint through time.  Each frame keeps a checkpoint (its tank
heads and warm start: flows, emitter flows, statuses); walking the frames in
reverse, the frame's polished forward is recomputed from the checkpoint,
which leaves its terminal factor in the plan, and one wds_adjoint launch
turns dL/d(heads, flows, emitter flows) of the frame, plus the tank-volume
sensitivity carried from later frames, into dL/d(demand of the frame's
pattern period, reservoir heads, Ke, r) and dL/d(tank heads) carried to
earlier frames.  A time step is a constant of the backward pass (it moves
only at the rounding of the tank fill time), and a clamped update carries
nothing.  No factor of any frame is stored.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .autodiff import _adjoint_guards, _clamp_grh, _clamp_rhs
from .solver import GGASolver, _check_info_flags, _not_pd_hint

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
        self.hmax = f(net.tank_hmax)
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


def _step_forward(s, d, rh, ke, r, B, max_iter, acc, polish, q0, e0, S0=None):
    o = s.run(d, rh, ke, r, B, max_iter, acc, True, polish, q0=q0, e0=e0, S0=S0)
    info = o["info"]
    _check_info_flags(s, info)
    if bool((info != 0).any()):
        bad = torch.nonzero(info != 0).flatten().tolist()
        if bool((info & _lib.INFO_NOT_PD).any()):
            raise RuntimeError("eps: the node matrix of scenarios %s is not positive definite%s"
                               % (bad[:8], _not_pd_hint(s)))
        raise RuntimeError("eps: scenarios %s did not converge (relerr=%s > accuracy=%g)"
                           % (bad[:8], [float(o["relerr"][b]) for b in bad[:4]], acc))
    return o


def _round_c(x):
    """ROUND of the reference (types.h:103): (int)(x + .5) or (int)(x - .5)."""
    return np.where(x >= 0.0, np.trunc(x + 0.5), np.trunc(x - 0.5))


class _Clock:
    """EpsDriver's per-scenario clock (nexthyd / timestep, dgga/eps.py:
    262-276, 211-229, 278-291, 332-350) on the host, in float64 and integer
    seconds as the reference: the time step after a frame and the tank
    update (explicit Euler with the one-second look-ahead clamp)."""

    def __init__(self, tk, h0, dur, hstep, pstep, rstep, pstart):
        self.tk = tk
        B = h0.shape[0]
        self.dur, self.hstep, self.pstep, self.rstep, self.pstart = dur, hstep, pstep, rstep, pstart
        self.htime = np.zeros(B, dtype=np.int64)
        self.rtime = np.full(B, rstep, dtype=np.int64)
        self.done = np.zeros(B, dtype=bool)
        self.area = tk.area.cpu().numpy()
        self.hmin = tk.hmin.cpu().numpy()
        self.hmax = tk.hmax.cpu().numpy()
        self.vmin = tk.vmin.cpu().numpy()
        self.vmax = tk.vmax.cpu().numpy()
        self.h = np.array(h0, dtype=np.float64)    # tank heads of the next frame
        self.v = self.vmin + (self.h - self.hmin) * self.area   # tank volumes (the state)

    def period(self, P):
        return np.minimum((self.htime + self.pstart) // self.pstep, P - 1)

    def advance(self, qnet):
        """After the frames at self.htime: the time steps and clamped masks;
        self.h / self.v move to the next frame.  Scenarios at the end get step
        0 and are done."""
        h, v = self.h, self.v
        B, nt = h.shape
        last = self.htime >= self.dur
        tstep = np.full(B, self.hstep, dtype=np.int64)
        t = ((self.htime + self.pstart) // self.pstep + 1) * self.pstep - self.htime
        tstep = np.where((t > 0) & (t < tstep), t, tstep)
        t = self.rtime - self.htime
        tstep = np.where((t > 0) & (t < tstep), t, tstep)
        for j in range(nt):  # tanktimestep: tanks in order
            qn = qnet[:, j]
            fill = (qn > 0.0) & (h[:, j] < self.hmax[j])
            empty = ~fill & (qn < 0.0) & (h[:, j] > self.hmin[j])
            dv = np.where(fill, self.vmax[j] - v[:, j], self.vmin[j] - v[:, j])
            with np.errstate(divide="ignore", invalid="ignore"):
                tt = _round_c(np.where(np.abs(qn) > 1e-6, dv / qn, 0.0)).astype(np.int64)
            use = (np.abs(qn) > 1e-6) & (fill | empty) & (tt > 0) & (tt < tstep)
            tstep = np.where(use, tt, tstep)
        tstep = np.where(last | self.done, 0, tstep)
        v2 = v + qnet * tstep[:, None]
        hi = v2 + qnet >= self.vmax
        lo = ~hi & (v2 - qnet <= self.vmin)
        v2 = np.where(hi, self.vmax, np.where(lo, self.vmin, v2))
        moving = (tstep > 0)[:, None]
        self.v = np.where(moving, v2, v)
        self.h = np.where(moving, self.hmin + (v2 - self.vmin) / self.area, h)
        clamped = (hi | lo) & moving
        self.htime = np.where(self.done, self.htime, self.htime + tstep)
        self.rtime = np.where(self.htime >= self.rtime, self.rtime + self.rstep, self.rtime)
        self.done = self.done | last
        return tstep, clamped


class EpsSM100(torch.autograd.Function):
    """(demand[P,B,N], res_head[B,N], tank_h0[B,nt], ke[B or 1,N],
    r_hw[B or 1,L], solver, clock options, accuracy, max_iter, polish_steps)
    -> (head[F,B,N], flow[F,B,L], emitter[F,B,N], tank_head[F,B,nt],
    t_sec[F,B], valid[F,B], status[F,B,L])."""

    @staticmethod
    def forward(ctx, demand, res_head, tank_h0, ke, r_hw, solver, clock, accuracy, max_iter,
                polish_steps, max_frames):
        s = solver
        tk = _Tanks(s)
        P, B, N = demand.shape
        L = s.L
        dev = s.device
        d_all = demand.detach().contiguous()
        rh0 = res_head.detach().contiguous()
        ke_t = ke.detach().contiguous()
        r_t = r_hw.detach().contiguous()
        ck = _Clock(tk, tank_h0.detach().cpu().numpy().astype(np.float64), *clock)
        bidx = torch.arange(B, device=dev)
        frames = []
        q0 = e0 = S0 = None
        while not ck.done.all():
            if len(frames) >= max_frames:
                raise RuntimeError("eps_solve: more than %d frames" % max_frames)
            valid = ~ck.done
            per = ck.period(P)
            d = d_all[torch.as_tensor(per, device=dev), bidx].contiguous()
            ht = torch.as_tensor(ck.h, device=dev)
            rh = rh0.clone()
            rh[:, tk.node] = ht
            o = _step_forward(s, d, rh, ke_t, r_t, B, max_iter, accuracy, polish_steps,
                              q0, e0, S0)
            _adjoint_guards(s, o["flow"], o["status"], allow_clamp=True)
            qnet = tk.inflow(o["flow"], o["status"])
            t_now = ck.htime.copy()
            tstep, clamped = ck.advance(qnet.cpu().numpy())
            vt = torch.as_tensor(valid, device=dev)
            fr = dict(head=o["head"], flow=o["flow"], emit=o["emit"], status=o["status"],
                      tank=ht, t=np.where(valid, t_now, -1), valid=valid, per=per,
                      dt=tstep, clamped=clamped,
                      opened=o["status"].index_select(1, tk.k) > ST_CLOSED,
                      warm=(q0, e0, S0), vt=vt)
            frames.append(fr)
            # the next frame starts where this one ended; finished scenarios keep
            # their last state (their padding frames are not outputs)
            q0 = o["flow"].contiguous() if q0 is None else \
                torch.where(vt[:, None], o["flow"], q0).contiguous()
            e0 = o["emit"].contiguous() if e0 is None else \
                torch.where(vt[:, None], o["emit"], e0).contiguous()
            S0 = o["status"].contiguous() if S0 is None else \
                torch.where(vt[:, None], o["status"], S0).contiguous()
        F = len(frames)
        z = lambda *sh, dt=torch.float64: torch.zeros(*sh, dtype=dt, device=dev)
        heads, flows, emits = z(F, B, N), z(F, B, L), z(F, B, N)
        tank_heads, status = z(F, B, tk.nt), z(F, B, L, dt=torch.int8)
        for f, fr in enumerate(frames):
            m = fr["vt"][:, None]
            heads[f] = torch.where(m, fr["head"], 0.0)
            flows[f] = torch.where(m, fr["flow"], 0.0)
            emits[f] = torch.where(m, fr["emit"], 0.0)
            tank_heads[f] = torch.where(m, fr["tank"], 0.0)
            status[f] = torch.where(m, fr["status"], torch.zeros_like(fr["status"]))
        t_sec = torch.as_tensor(np.stack([fr["t"] for fr in frames]), device=dev)
        valid = torch.as_tensor(np.stack([fr["valid"] for fr in frames]), device=dev)
        for fr in frames:   # the checkpoints keep only the warm start and the clock
            for k in ("head", "flow", "emit", "status"):
                fr.pop(k)
        ctx.frames = frames
        ctx.save_for_backward(d_all, rh0, ke_t, r_t)
        ctx.solver, ctx.tk = s, tk
        ctx.args = (float(accuracy), int(max_iter), int(polish_steps))
        ctx.kedim, ctx.rdim = ke.shape[0], r_hw.shape[0]
        ctx.mark_non_differentiable(t_sec, valid, status)
        return heads, flows, emits, tank_heads, t_sec, valid, status

    @staticmethod
    def backward(ctx, gH, gQ, gE, gT, _gt, _gv, _gs):
        if torch.is_grad_enabled():
            raise NotImplementedError("the extended-period adjoint is first order only")
        s, tk, frames = ctx.solver, ctx.tk, ctx.frames
        d_all, rh0, ke_t, r_t = ctx.saved_tensors
        acc, max_iter, polish = ctx.args
        P, B, N = d_all.shape
        F = len(frames)
        L = s.L
        dev = s.device
        z = lambda *sh: torch.zeros(*sh, dtype=torch.float64, device=dev)
        gH = z(F, B, N) if gH is None else gH.to(torch.float64)
        gQ = z(F, B, L) if gQ is None else gQ.to(torch.float64)
        gE = z(F, B, N) if gE is None else gE.to(torch.float64)
        gT = z(F, B, tk.nt) if gT is None else gT.to(torch.float64)
        g_dem = z(P, B, N)
        g_rh = z(B, N)
        g_ke = z(B, N)
        g_r = z(B, L)
        gV = z(B, tk.nt)                           # dL/dV after the frame in hand
        bidx = torch.arange(B, device=dev)
        for f in range(F - 1, -1, -1):
            fr = frames[f]
            vt = fr["vt"]
            dt = torch.as_tensor(fr["dt"], dtype=torch.float64, device=dev)[:, None]
            free = ~torch.as_tensor(fr["clamped"], device=dev)
            gqnet = torch.where(free & vt[:, None], gV * dt, 0.0)   # dL/dQnet of the frame
            gV = torch.where(free, gV, 0.0)
            m = vt[:, None]
            gq = torch.where(m, gQ[f], 0.0)
            gq.index_add_(1, tk.k, gqnet.index_select(1, tk.j) * tk.sign * fr["opened"])
            per = torch.as_tensor(fr["per"], device=dev)
            d = d_all[per, bidx].contiguous()
            rh = rh0.clone()
            rh[:, tk.node] = fr["tank"]
            q0, e0, S0 = fr["warm"]
            o = _step_forward(s, d, rh, ke_t, r_t, B, max_iter, acc, polish,
                              None if q0 is None else q0.contiguous(),
                              None if e0 is None else e0.contiguous(),
                              None if S0 is None else S0.contiguous())
            gHt = torch.where(m, gH[f], 0.0).contiguous()
            gEt = torch.where(m, gE[f], 0.0).contiguous()
            gq = gq.contiguous()
            # constant-HP pumps on their clamp branch: Woodbury on the kept factor
            clamp = _adjoint_guards(s, o["flow"], o["status"], allow_clamp=True)
            fix = None
            if clamp is not None:
                gHt, fix = _clamp_rhs(s, o["plan"], B, clamp, gHt, gq, gEt,
                                      torch.cuda.current_stream(dev).cuda_stream)
            gd, grh, gke, gr = _adjoint_launch(s, o["plan"], B, gHt, gq, gEt)
            if fix is not None:
                _clamp_grh(fix, gq, gd, grh)
            gd, grh = torch.where(m, gd, 0.0), torch.where(m, grh, 0.0)
            gke, gr = torch.where(m, gke, 0.0), torch.where(m, gr, 0.0)
            g_dem.index_put_((per, bidx), gd, accumulate=True)
            g_rh += grh
            g_ke += gke
            g_r += gr
            gV = gV + torch.where(m, grh.index_select(1, tk.node) + gT[f], 0.0) / tk.area
        g_rh[:, tk.node] = 0.0                     # tank entries of res_head are not used
        g_h0 = gV * tk.area
        g_ke = g_ke.sum(0, keepdim=True) if ctx.kedim == 1 else g_ke
        g_r = g_r.sum(0, keepdim=True) if ctx.rdim == 1 else g_r
        return g_dem, g_rh, g_h0, g_ke, g_r, None, None, None, None, None, None


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
              duration=None, hstep=3600, pstep=3600, rstep=None, pstart=0, accuracy=1e-6,
              max_iter=200, polish_steps=3, max_frames=100000):
    """Batched extended-period run on EpsDriver's clock.

    demand [P,B,N] (cfs) per pattern period (period p covers [p pstep,
    (p + 1) pstep) after pstart); res_head [B,N] or [N] fixed heads (ft; tank
    entries are ignored, default: the network's reservoir heads); tank_h0
    [B,nt] or [nt] initial tank heads (default net.tank_h0); ke [N] or [B,N];
    r_hw [L] or [B,L]; duration (s, default (P - 1) pstep), hstep, pstep,
    rstep (default pstep), pstart: the clock of EpsDriver (eps.py:48-63).
    Returns dict(head [F,B,N], flow [F,B,L], emitter [F,B,N], tank_head
    [F,B,nt] (the tank heads the frame was solved with), t_sec [F,B] (-1 on
    padding), valid [F,B], status [F,B,L]), differentiable w.r.t. demand,
    res_head, tank_h0, ke and r_hw (1-D parameters receive the batch-summed
    gradient)."""
    s = solver
    dev = s.device
    if s.net.tank_node is None or len(s.net.tank_node) == 0:
        raise ValueError("eps_solve: the network has no tanks")
    t = lambda x: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    demand = t(demand)
    if demand.dim() != 3 or demand.shape[2] != s.N:
        raise ValueError("eps_solve: demand must be [P, B, N]")
    P, B, N = demand.shape
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
    dur = (P - 1) * int(pstep) if duration is None else int(duration)
    clock = (dur, int(hstep), int(pstep), int(pstep if rstep is None else rstep), int(pstart))
    head, flow, emit, tank_head, t_sec, valid, status = EpsSM100.apply(
        demand, res_head, tank_h0, ke, r_hw, s, clock, float(accuracy), int(max_iter),
        int(polish_steps), int(max_frames))
    return dict(head=head, flow=flow, emitter=emit, tank_head=tank_head, t_sec=t_sec,
                valid=valid, status=status)
