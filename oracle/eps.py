"""CPU oracle of the batched extended-period run and its adjoint through time.

TEST INFRASTRUCTURE ONLY (imported by tests/).  The reference has no batched
or differentiable extended-period path, so this oracle is a composition:
each step is the oracle's implicit steady solve (oracle.gga.Model.implicit,
warm started from the previous step as GGASolver.solve(q0=, e0=) does,
dgga/solver.py:2876-2887), followed by the reference's tank update
(EpsDriver._tanklevels dgga/eps.py:278-291, _tankgrade :91-95, tank net inflow
as in solver.py:2063-2073).  The backward pass walks the steps in reverse with
Model.backward on each step's kept state.  The step semantics (tank update,
signs, clamp) are pinned against the reference's own EpsDriver by
tests/test_eps_oracle.py (fixture tests/golden/eps_ref.npz).
"""
from __future__ import annotations

import numpy as np

from .gga import Model, CLOSED


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

    def inflow(self, q, S):
        B = q.shape[0]
        out = np.zeros((B, self.tnode.size))
        w = q[:, self.k] * (S[:, self.k] > CLOSED) * self.sign
        for c in range(self.k.size):
            out[:, self.j[c]] += w[:, c]
        return out

    def run(self, demand, res_head, tank_h0, ke=None, r=None, dt=3600.0, accuracy=1e-6,
            max_iter=200, polish_steps=3):
        """demand [T,B,N]; res_head [B,N]; tank_h0 [B,nt].  Returns the
        trajectory and the per-step states for backward()."""
        T, B, N = demand.shape
        h = np.array(tank_h0, dtype=np.float64)
        v = self.vmin + (h - self.hmin) * self.area
        out = dict(head=[], flow=[], emitter=[], tank_head=[h.copy()], iters=[])
        states, clamped = [], []
        q0 = e0 = None
        for t in range(T):
            rh = np.array(res_head, dtype=np.float64)
            rh[:, self.tnode] = h
            o, st = self.m.implicit(demand[t], rh, ke=ke, r=r, accuracy=accuracy,
                                    max_iter=max_iter, polish_steps=polish_steps,
                                    q0=q0, e0=e0)
            out["head"].append(o["head_ft"]); out["flow"].append(o["flow_cfs"])
            out["emitter"].append(o["emitter_cfs"]); out["iters"].append(o["iters"])
            qnet = self.inflow(o["flow_cfs"], o["status"])
            v = v + qnet * dt
            hi = v + qnet >= self.vmax
            lo = ~hi & (v - qnet <= self.vmin)
            v = np.where(hi, self.vmax, np.where(lo, self.vmin, v))
            h = self.hmin + (v - self.vmin) / self.area
            out["tank_head"].append(h.copy())
            states.append((st, o["status"]))
            clamped.append(hi | lo)
            q0, e0 = o["flow_cfs"], o["emitter_cfs"]
        res = {k: np.asarray(x) for k, x in out.items()}
        res["_states"], res["_clamped"], res["_dt"] = states, clamped, dt
        return res

    def backward(self, run, gH, gQ, gE, gT):
        """Adjoint through time; returns (g_demand [T,B,N], g_res_head [B,N],
        g_tank_h0 [B,nt], g_ke [B,N], g_r [B,L])."""
        T, B, N = gH.shape
        dt = run["_dt"]
        g_dem = np.zeros((T, B, N))
        g_rh = np.zeros((B, N))
        g_ke = np.zeros((B, N))
        g_r = np.zeros((B, self.m.L))
        gV = gT[T] / self.area
        for t in range(T - 1, -1, -1):
            st, S = run["_states"][t]
            free = ~run["_clamped"][t]
            gqnet = np.where(free, gV * dt, 0.0)
            gV = np.where(free, gV, 0.0)
            gq = np.array(gQ[t], dtype=np.float64)
            opened = S[:, self.k] > CLOSED
            for c in range(self.k.size):
                gq[:, self.k[c]] += gqnet[:, self.j[c]] * self.sign[c] * opened[:, c]
            gd, grh, gke, gr = self.m.backward(st, gH[t], gq, gE[t])
            g_dem[t] = gd
            g_rh += grh
            g_ke += gke
            g_r += gr
            gV = gV + (grh[:, self.tnode] + gT[t]) / self.area
        g_rh[:, self.tnode] = 0.0
        return g_dem, g_rh, gV * self.area, g_ke, g_r
