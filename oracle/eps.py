"""CPU oracle of the batched extended-period run and its adjoint through time.

TEST INFRASTRUCTURE ONLY (imported by tests/).  The reference has no batched
or differentiable extended-period path, so this oracle is a composition:
each frame is the oracle's implicit steady solve (oracle.gga.Model.implicit,
warm started from the previous frame's flows, emitter flows and statuses as
EpsDriver.run does, dgga/eps.py:366-373), followed by the reference's time
step (EpsDriver._timestep :262-276: the hydraulic step shortened at pattern
boundaries, report times and tank fill/empty times, tanktimestep :211-229)
and tank update (_tanklevels :278-291, _tankgrade :91-95, tank net inflow as
in solver.py:2063-2073).  The backward pass walks the steps in reverse with
Model.backward on each step's kept state.  The step semantics (tank update,
signs, clamp) are pinned against the reference's own EpsDriver by
tests/test_eps_oracle.py (fixture tests/golden/eps_ref.npz).
"""
from __future__ import annotations

import numpy as np

from .gga import Model, CLOSED

QZERO = 1e-6  # dgga/solver.py QZERO


class EpsOracle:
    def __init__(self, net):
        self.m = Model(net)
        self.net = net
        tn = np.asarray(net.tank_node, dtype=np.int64)
        self.tnode = tn
        pos = {int(n): j for j, n in enumerate(tn)}
        ks, js, sg = [], [], []
        for k in range(self.m.L):
            a, b = int(net.link_n1[k]), int(net.link_n2[k])
            if a in pos:
                ks.append(k); js.append(pos[a]); sg.append(-1.0)
            if b in pos:
                ks.append(k); js.append(pos[b]); sg.append(1.0)
        self.k = np.asarray(ks, dtype=np.int64)
        self.j = np.asarray(js, dtype=np.int64)
        self.sign = np.asarray(sg)
        self.area = np.asarray(net.tank_area, dtype=np.float64)
        self.hmin = np.asarray(net.tank_hmin, dtype=np.float64)
        self.vmin = np.asarray(net.tank_vmin, dtype=np.float64)
        self.vmax = np.asarray(net.tank_vmax, dtype=np.float64)
        self.hmax = np.asarray(net.tank_hmax, dtype=np.float64)

    def inflow(self, q, S):
        B = q.shape[0]
        out = np.zeros((B, self.tnode.size))
        w = q[:, self.k] * (S[:, self.k] > CLOSED) * self.sign
        for c in range(self.k.size):
            out[:, self.j[c]] += w[:, c]
        return out

    def tank_time(self, tstep, h, qnet, v):
        """tanktimestep (EpsDriver._tanktimestep, dgga/eps.py:211-229): the
        rounded time to the first tank filling or emptying, if shorter."""
        for j in range(self.tnode.size):
            qn = qnet[j]
            if abs(qn) <= QZERO:
                continue
            if qn > 0.0 and h[j] < self.hmax[j]:
                dv = self.vmax[j] - v[j]
            elif qn < 0.0 and h[j] > self.hmin[j]:
                dv = self.vmin[j] - v[j]
            else:
                continue
            x = dv / qn
            t = int(x + 0.5) if x >= 0.0 else int(x - 0.5)   # ROUND (types.h:103)
            if 0 < t < tstep:
                tstep = t
        return tstep

    def run(self, demand, res_head, tank_h0, ke=None, r=None, duration=None, hstep=3600,
            pstep=3600, rstep=None, pstart=0, accuracy=1e-6, max_iter=200, polish_steps=3):
        """EpsDriver.run's frames (dgga/eps.py:356-411) per scenario: frame at
        Htime, then the time step min(Hstep, pattern boundary, report time,
        tank fill/empty time) and the tank update (eps.py:262-276, 211-229,
        278-291); link flows, emitter flows and statuses carry from frame to
        frame.  demand [P,B,N] per pattern period; res_head [B,N]; tank_h0
        [B,nt].  Returns per scenario lists of frames and their states for
        backward()."""
        P, B, N = demand.shape
        dur = (P - 1) * pstep if duration is None else int(duration)
        rstep = pstep if rstep is None else int(rstep)
        runs = []
        for b in range(B):
            h = np.array(tank_h0[b], dtype=np.float64)
            v = self.vmin + (h - self.hmin) * self.area
            htime, rtime = 0, rstep
            q0 = e0 = S0 = None
            fr = dict(t=[], head=[], flow=[], emitter=[], status=[], tank_head=[], iters=[],
                      state=[], dt=[], clamped=[], period=[], warm=[])
            while True:
                p = min((htime + pstart) // pstep, P - 1)
                rh = np.array(res_head[b], dtype=np.float64)
                rh[self.tnode] = h
                kb = None if ke is None else np.atleast_2d(ke)[min(b, np.atleast_2d(ke).shape[0] - 1)]
                rb = None if r is None else np.atleast_2d(r)[min(b, np.atleast_2d(r).shape[0] - 1)]
                o, st = self.m.implicit(demand[p, b][None], rh[None], ke=kb, r=rb,
                                        accuracy=accuracy, max_iter=max_iter,
                                        polish_steps=polish_steps, q0=q0, e0=e0, S0=S0)
                fr["warm"].append((q0, e0, S0))
                fr["t"].append(htime); fr["period"].append(p)
                fr["head"].append(o["head_ft"][0]); fr["flow"].append(o["flow_cfs"][0])
                fr["emitter"].append(o["emitter_cfs"][0]); fr["status"].append(o["status"][0])
                fr["tank_head"].append(h.copy()); fr["iters"].append(int(o["iters"][0]))
                fr["state"].append((st, o["status"]))
                qnet = self.inflow(o["flow_cfs"], o["status"])[0]
                if htime >= dur:
                    fr["dt"].append(0); fr["clamped"].append(np.zeros(self.tnode.size, bool))
                    break
                tstep = hstep
                t = ((htime + pstart) // pstep + 1) * pstep - htime   # pattern boundary
                if 0 < t < tstep:
                    tstep = t
                t = rtime - htime                                      # report time
                if 0 < t < tstep:
                    tstep = t
                tstep = self.tank_time(tstep, h, qnet, v)
                v = v + qnet * tstep
                hi = v + qnet >= self.vmax
                lo = ~hi & (v - qnet <= self.vmin)
                v = np.where(hi, self.vmax, np.where(lo, self.vmin, v))
                h = self.hmin + (v - self.vmin) / self.area
                fr["dt"].append(tstep); fr["clamped"].append(hi | lo)
                htime += tstep
                if htime >= rtime:
                    rtime += rstep
                q0, e0, S0 = o["flow_cfs"], o["emitter_cfs"], o["status"]
            runs.append(fr)
        return runs

    def backward(self, runs, gH, gQ, gE, gT, P):
        """Adjoint through time of run(): gH/gQ/gE/gT are per scenario lists
        of [F_b, .] arrays (frame heads, flows, emitter flows, tank heads).
        Returns (g_demand [P,B,N], g_res_head [B,N], g_tank_h0 [B,nt],
        g_ke [B,N], g_r [B,L]).  A time step is a constant (it changes only
        at the rounding of tanktimestep), a clamped tank update carries
        nothing."""
        B = len(runs)
        N, L = self.m.N, self.m.L
        g_dem = np.zeros((P, B, N))
        g_rh = np.zeros((B, N))
        g_ke = np.zeros((B, N))
        g_r = np.zeros((B, L))
        g_h0 = np.zeros((B, self.tnode.size))
        for b, fr in enumerate(runs):
            F = len(fr["t"])
            gV = np.zeros(self.tnode.size)
            for f in range(F - 1, -1, -1):
                st, S = fr["state"][f]
                dt = fr["dt"][f]
                free = ~fr["clamped"][f]
                gqnet = np.where(free, gV * dt, 0.0)
                gV = np.where(free, gV, 0.0)
                gq = np.array(gQ[b][f], dtype=np.float64)[None].copy()
                opened = S[:, self.k] > CLOSED
                for c in range(self.k.size):
                    gq[:, self.k[c]] += gqnet[self.j[c]] * self.sign[c] * opened[:, c]
                gd, grh, gke, gr = self.m.backward(st, np.asarray(gH[b][f])[None], gq,
                                                   np.asarray(gE[b][f])[None])
                g_dem[fr["period"][f], b] += gd[0]
                g_rh[b] += grh[0]
                g_ke[b] += gke[0]
                g_r[b] += gr[0]
                gV = gV + (grh[0, self.tnode] + np.asarray(gT[b][f])) / self.area
            g_h0[b] = gV * self.area
        g_rh[:, self.tnode] = 0.0
        return g_dem, g_rh, g_h0, g_ke, g_r
