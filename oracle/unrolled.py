"""CPU oracle of the unrolled-K GGA and of its reverse-mode gradient.

TEST INFRASTRUCTURE ONLY (imported by tests/ alone).  Restates
`solve_unrolled` (dgga/autodiff.py:1357-1664): K GGA iterations with no
convergence test and the link statuses frozen, on networks of pipes, check-
valve pipes, TCVs and pumps with emitters and fixed heads.  The reference
differentiates that loop with torch autograd; here the gradient w.r.t.
demand, fixed heads, emitter Ke and pipe resistance comes from an explicit
reverse pass: every iteration's linear solve transposed (the node matrix is
symmetric), and each coefficient differentiated on the branch the forward
took, as autograd differentiates `torch.where` / `clamp_min` (a clamped
quantity has zero derivative; |q| is q * sgn with sgn constant).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from .gga import CBIG, CLOSED, CSMALL, Model

__all__ = ["Unrolled"]


class Unrolled:
    def __init__(self, model: Model):
        self.m = model

    # ------------------------------------------------------------ derivatives
    def link_derivs(self, q, r, S):
        """P, Y of every link and dP/dq, dY/dq, dP/dr, dY/dr on the branch
        taken (pipes solver.py:2176-2201, TCV :2203-2219, pumps :2221-2326 as
        restated in solve_unrolled; closed and NOCURVE links: P const, Y = q)."""
        m = self.m
        P, Y, closed = m.headloss_PY(q, r, S)
        sgn = np.where(q < 0, -1.0, 1.0)
        qa = q * sgn
        z = np.zeros_like(q)
        Pq, Yq, Pr, Yr = z.copy(), z.copy(), z.copy(), z.copy()
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            # pipes: hg = hexp r qa^(hexp-1) (RQtol clamp), hl = hg qa / hexp, + Km qa^2
            n = m.hexp
            qc = np.maximum(qa, 1e-30)
            hg0 = n * r * qc ** (n - 1.0)
            lin = hg0 < m.rqtol
            live = qa > 1e-30
            hg = np.where(lin, m.rqtol, hg0)
            hl = np.where(lin, hg * qa, hg * qa / n)
            dhg = np.where(lin | ~live, 0.0, n * (n - 1.0) * r * qc ** (n - 2.0))
            dhl = np.where(lin, m.rqtol, dhg * qa / n + hg / n)
            dhg_r = np.where(lin, 0.0, n * qc ** (n - 1.0))
            dhl_r = dhg_r * qa / n
            mp = m.km > 0.0
            hl = np.where(mp, hl + m.km * qa * qa, hl)
            dhl = np.where(mp, dhl + 2.0 * m.km * qa, dhl)
            hg = np.where(mp, hg + 2.0 * m.km * qa, hg)
            dhg = np.where(mp, dhg + 2.0 * m.km, dhg)
            # P = 1/hg, Y = hl sgn / hg; d(qa)/dq = sgn
            pq = -dhg * sgn / (hg * hg)
            yq = (dhl * hg - hl * dhg) / (hg * hg)
            pr = -dhg_r / (hg * hg)
            yr = sgn * (dhl_r * hg - hl * dhg_r) / (hg * hg)
            pipe = ~m.is_tcv & ~m.is_pump
            Pq, Yq = np.where(pipe, pq, Pq), np.where(pipe, yq, Yq)
            Pr, Yr = np.where(pipe, pr, Pr), np.where(pipe, yr, Yr)
            # TCV: hg = 2 Km qa (RQtol clamp), hl = q hg / 2 (or q RQtol)
            km = m.km_tcv
            hgv0 = 2.0 * km * qa
            linv = hgv0 < m.rqtol
            hgv = np.where(linv, m.rqtol, hgv0)
            dhgv = np.where(linv, 0.0, 2.0 * km * sgn)
            hlv = np.where(linv, q * hgv, q * hgv / 2.0)
            dhlv = np.where(linv, hgv, (hgv + q * dhgv) / 2.0)
            kp = km > 0.0
            tq_p = np.where(kp, -dhgv / (hgv * hgv), 0.0)
            tq_y = np.where(kp, (dhlv * hgv - hlv * dhgv) / (hgv * hgv), 1.0)
            Pq = np.where(m.is_tcv, tq_p, Pq)
            Yq = np.where(m.is_tcv, tq_y, Yq)
            if m.n_pumps:
                pp, py = self._pump_derivs(q, sgn, qa)
                Pq = np.where(m.is_pump, pp, Pq)
                Yq = np.where(m.is_pump, py, Yq)
        # closed branch: P = 1/CBIG, Y = q
        Pq = np.where(closed, 0.0, Pq)
        Yq = np.where(closed, 1.0, Yq)
        Pr = np.where(closed | ~(~m.is_tcv & ~m.is_pump), 0.0, Pr)
        Yr = np.where(closed | ~(~m.is_tcv & ~m.is_pump), 0.0, Yr)
        return P, Y, Pq, Yq, Pr, Yr

    def _pump_derivs(self, q, sgn, qa):
        """dP/dq, dY/dq of pumps on the branch taken (solve_unrolled's pump
        formulas, dgga/autodiff.py:1535-1585; a CUSTOM curve's segment is
        chosen from the detached flow, so its H0 and R are constants)."""
        m = self.m
        spc = np.maximum(m.speed, 1e-12)
        h0e = spc * spc * m.p_h0
        re = m.p_r * spc ** (2.0 - m.p_n)
        # CONST_HP: hg = -re / qa^2 clamped to [RQtol, CBIG]; hl = re / q or -hg q
        qa2 = np.maximum(qa * qa, 1e-30)
        raw = -re / qa2
        big, sml = raw > CBIG, raw < m.rqtol
        hg_c = np.where(big, CBIG, np.where(sml, m.rqtol, raw))
        dhg_c = np.where(big | sml | (qa * qa < 1e-30), 0.0, 2.0 * re / (qa2 * qa2) * qa * sgn)
        qcc = sgn * np.maximum(qa, 1e-30)
        hl_c = np.where(big | sml, -hg_c * q, re / qcc)
        dhl_c = np.where(big | sml, -hg_c, np.where(qa > 1e-30, -re / (qcc * qcc), 0.0))
        # POWER_FUNC: hg = n re qa^(n-1) (RQtol clamp); hl = h0 + hg q / n (or + RQtol q)
        n = m.p_n
        qc = np.maximum(qa, 1e-30)
        raw_p = n * re * qc ** (n - 1.0)
        sml_p = raw_p < m.rqtol
        hg_p = np.where(sml_p, m.rqtol, raw_p)
        dhg_p = np.where(sml_p | (qa <= 1e-30), 0.0, n * (n - 1.0) * re * qc ** (n - 2.0) * sgn)
        nn = np.maximum(n, 1e-30)
        hl_p = np.where(sml_p, h0e + hg_p * q, h0e + hg_p * q / nn)
        dhl_p = np.where(sml_p, hg_p, (dhg_p * q + hg_p) / nn)
        # linear n = 1: hg = re, hl = h0 + re q
        hg_p = np.where(m.p_lin, re, hg_p)
        dhg_p = np.where(m.p_lin, 0.0, dhg_p)
        hl_p = np.where(m.p_lin, h0e + re * q, hl_p)
        dhl_p = np.where(m.p_lin, re, dhl_p)
        hg = np.where(m.p_chp, hg_c, hg_p)
        dhg = np.where(m.p_chp, dhg_c, dhg_p)
        hl = np.where(m.p_chp, hl_c, hl_p)
        dhl = np.where(m.p_chp, dhl_c, dhl_p)
        for k, (cx, cy) in m.curves.items():   # frozen segment: hg const, hl = H0 w^2 + hg q
            s = max(m.speed[k], 1e-12)
            qq = (np.abs(q[:, k]) / s) * m.ucf_flow
            idx = np.searchsorted(cx, qq, side="left")
            k2 = np.minimum(np.maximum(idx, 1), cx.size - 1)
            k1 = k2 - 1
            rc = (cy[k2] - cy[k1]) / (cx[k2] - cx[k1])
            h0c = (cy[k1] - rc * cx[k1]) / m.ucf_head
            rc = rc * m.ucf_flow / m.ucf_head
            hg[:, k] = (-rc) * s
            dhg[:, k] = 0.0
            hl[:, k] = (-h0c) * (s * s) + hg[:, k] * q[:, k]
            dhl[:, k] = hg[:, k]
        pq = -dhg / (hg * hg)
        yq = (dhl * hg - hl * dhg) / (hg * hg)
        pq = np.where(m.p_nocurve, 0.0, pq)
        yq = np.where(m.p_nocurve, 1.0, yq)
        return pq, yq

    def emitter_derivs(self, e, ke):
        """hle, hge of the emitters and their derivatives in e and Ke
        (solver.py:2368-2377 as in solve_unrolled)."""
        m = self.m
        kea = np.maximum(ke, CSMALL)
        dkea = (ke > CSMALL).astype(float)
        ea = np.maximum(np.abs(e), 1e-30)
        live = np.abs(e) > 1e-30
        sg = np.sign(e)
        hg0 = m.qexp * kea * ea ** (m.qexp - 1.0)
        lin = hg0 < m.rqtol
        hge = np.where(lin, m.rqtol, hg0)
        hle = np.where(lin, hge * e, hge * e / m.qexp)
        hge_e = np.where(lin | ~live, 0.0, m.qexp * (m.qexp - 1.0) * kea * ea ** (m.qexp - 2.0) * sg)
        hge_k = np.where(lin, 0.0, m.qexp * ea ** (m.qexp - 1.0) * dkea)
        hle_e = np.where(lin, m.rqtol, (hge_e * e + hge) / m.qexp)
        hle_k = np.where(lin, 0.0, hge_k * e / m.qexp)
        return hle, hge, hle_e, hge_e, hle_k, hge_k

    # ---------------------------------------------------------------- forward
    def forward(self, d, rh, ke=None, r=None, K=8, S=None, q0=None, e0=None):
        """K iterations from the initial flows (emitter flows 1), or from the
        warm start q0 [B or 1, L] / e0 [B or 1, N] of solve_unrolled
        (dgga/autodiff.py:1357-1360), with the statuses S frozen; returns the
        outputs and the record the reverse pass reads."""
        m = self.m
        d = np.atleast_2d(np.asarray(d, dtype=np.float64))
        B = d.shape[0]
        rh = np.broadcast_to(np.atleast_2d(np.nan_to_num(rh)), (B, m.N))
        ke = m.ke_default if ke is None else np.asarray(ke, dtype=np.float64)
        ke = np.broadcast_to(np.atleast_2d(ke), (B, m.N))
        r = m.r_hw if r is None else np.asarray(r, dtype=np.float64)
        r = np.broadcast_to(np.atleast_2d(r), (B, m.L))
        S = np.broadcast_to(m.S0 if S is None else np.asarray(S, dtype=np.int8), (B, m.L)).copy()
        ke_j, d_j = ke[:, m.junc], d[:, m.junc]
        em = (ke_j > 0.0).astype(float)
        q = np.broadcast_to(m.init_flow() if q0 is None else np.asarray(q0, dtype=np.float64),
                            (B, m.L)).copy()
        if e0 is None:
            e = em.copy()
        else:
            e0 = np.broadcast_to(np.atleast_2d(np.asarray(e0, dtype=np.float64)), (B, m.N))
            e = np.where(em > 0, e0[:, m.junc], 0.0)
        H = np.zeros((B, m.N))
        H[:, m.fixed] = rh[:, m.fixed]
        rec = []
        for _ in range(int(K)):
            P, Y, _ = m.headloss_PY(q, r, S)
            _, _, F, A, hle, hge, _ = m._assemble(P, Y, q, H, e, ke_j, d_j, S)
            Hj = m._chol_solve(A, F)
            Hn = H.copy()
            Hn[:, m.junc] = Hj
            dh = Hn[:, m.n1] - Hn[:, m.n2]
            dq = Y - P * dh
            hit = m.is_pump & m.p_chp & (dq > q)
            dq = np.where(hit, q / 2.0, dq)
            dqe = (hle - (Hj - m.el_j)) / hge
            rec.append(dict(q=q, e=e, H=Hn, A=A, hit=hit, dqe=dqe))
            q = q - dq
            e = e - em * dqe
            H = Hn
        emit = np.zeros((B, m.N))
        emit[:, m.junc] = e * em
        state = dict(rec=rec, r=r, ke_j=ke_j, em=em, S=S, rh=rh, B=B)
        return dict(head_ft=H, flow_cfs=q, emitter_cfs=emit), state

    # --------------------------------------------------------------- backward
    def backward(self, state, gH, gQ, gE):
        """dL/d(demand, fixed heads, Ke, r) [B,*] of the K-iteration map for
        the output adjoints gH [B,N], gQ [B,L], gE [B,N]."""
        m = self.m
        B, r, ke_j, em, S = state["B"], state["r"], state["ke_j"], state["em"], state["S"]
        Nj = m.Nj
        qb = np.array(gQ, dtype=np.float64)
        eb = np.asarray(gE, dtype=np.float64)[:, m.junc] * em
        gd = np.zeros((B, m.N))
        grh = np.zeros((B, m.N))
        gke = np.zeros((B, m.N))
        gr = np.zeros((B, m.L))
        m1, m2 = m.m1f, m.m2f
        for kk in range(len(state["rec"]) - 1, -1, -1):
            rc = state["rec"][kk]
            q, e, Hn, A, hit, dqe = rc["q"], rc["e"], rc["H"], rc["A"], rc["hit"], rc["dqe"]
            P, Y, Pq, Yq, Pr, Yr = self.link_derivs(q, r, S)
            hle, hge, hle_e, hge_e, hle_k, hge_k = self.emitter_derivs(e, ke_j)
            Hj = Hn[:, m.junc]
            dh = Hn[:, m.n1] - Hn[:, m.n2]
            # q' = q - dq (dq = q/2 on the constant-HP half step)
            qn = qb.copy()
            dqb = -qb
            qn = qn + np.where(hit, dqb / 2.0, 0.0)
            dqb = np.where(hit, 0.0, dqb)
            Yb = dqb.copy()
            Pb = -dqb * dh
            dhb = -dqb * P
            Hb = np.zeros((B, m.N))
            for b in range(B):
                np.add.at(Hb[b], m.n1, dhb[b])
                np.add.at(Hb[b], m.n2, -dhb[b])
            if kk == len(state["rec"]) - 1:
                Hb = Hb + gH
            # e' = e - em dqe, dqe = (hle - (Hj - el)) / hge
            en = eb.copy()
            dqeb = -em * eb
            hleb = dqeb / hge
            hgeb = -dqeb * dqe / hge
            Hjb = Hb[:, m.junc] - dqeb / hge
            grh += Hb * m.fixmask
            # H = A^{-1} F
            Fb = np.stack([sla.solve(A[b], Hjb[b], assume_a="pos") for b in range(B)])
            u = Fb[:, m.j1c] * m1 - Fb[:, m.j2c] * m2
            v = Hj[:, m.j1c] * m1 - Hj[:, m.j2c] * m2
            Pb += -u * v
            hgeb += em * Fb * Hj / (hge * hge)
            # F: link Y terms, fixed-head grounding, emitters, Xflow
            Yb += u
            for lk, row, src in ((m.lk_g1, m.g1_row, m.g1_src), (m.lk_g2, m.g2_row, m.g2_src)):
                if lk.size:
                    Pb[:, lk] += Fb[:, row] * Hn[:, src]
                    for b in range(B):
                        np.add.at(grh[b], src, Fb[b, row] * P[b, lk])
            hleb += em * Fb / hge
            hgeb += -em * Fb * (hle + m.el_j) / (hge * hge)
            qn += -u
            en += -em * Fb
            gd[:, m.junc] += -Fb
            # coefficients
            qn += Pb * Pq + Yb * Yq
            gr += Pb * Pr + Yb * Yr
            en += hleb * hle_e + hgeb * hge_e
            gke[:, m.junc] += hleb * hle_k + hgeb * hge_k
            qb, eb = qn, en
        return gd, grh, gke, gr
