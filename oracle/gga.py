"""CPU oracle: numpy restatement of the reference's batched GGA path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
module; it is used by tests/, by `__graft_entry__.smoke()` as the checker, and
by bench.py's CPU-baseline leg.  It restates, in plain numpy, the algorithm of

  * GGASolver.solve (mode="dense", assemble="csr", linear_solver="dense"),
    dgga/solver.py:2703-3212, including the batched status machine
    (_linkstatus_batch :697-739, _prvstatus_batch :914-947) and the batched
    PRV valve coefficients (_prvcoeffs_batch :850-912);
  * the link coefficient formulas _pipe_PY :2176, _tcv_PY :2203,
    _pump_PY :2221, _valve_PY_ml :834, _emitter_hloss :2368;
  * ImplicitGGASolveGPU (dgga/autodiff.py:1157-1312): the reduced Newton
    polish with Woodbury row replacement for ACTIVE PRVs
    (_adjgpu_polish :1053, _adjgpu_primal_solve :965) and the reduced
    adjoint (_adjgpu_node_solve :1107, backward :1246).

The linear solves are dense Cholesky plus two refinement steps, as in the
reference dense route.  The module is pinned against golden vectors produced
by the reference itself (tests/golden/*.npz, see tests/test_oracle_golden.py).
"""
from __future__ import annotations

import copy

import numpy as np
import scipy.linalg as sla

CSMALL, CBIG, BIG, TINY, MISSING = 1e-6, 1e8, 1e10, 1e-6, -1e10
QZERO, RQTOL, PI = 1e-6, 1e-7, 3.141592654
XHEAD, TEMPCLOSED, CLOSED, OPEN, ACTIVE, XFLOW, XFCV, XPRESSURE = range(8)
_CVPIPE, _PIPE, _PUMP, _PRV, _PSV, _PBV, _FCV, _TCV, _GPV = range(9)
MperFT, PSIperFT, KPAperPSI = 0.3048, 0.4333, 6.895
SI_FLOW = ("LPS", "LPM", "MLD", "CMH", "CMD")
FLOW_UCF = {"CFS": 1.0, "GPM": 448.831, "MGD": 0.64632, "IMGD": 0.5382,
            "AFD": 1.9837, "LPS": 28.317, "LPM": 1699.0, "MLD": 2.4466,
            "CMH": 101.94, "CMD": 2446.6}


def _scatter(n_rows, idx, vals):
    """Sequential scatter-add over the last axis (np.add.at is sequential in
    index order, like a CPU scatter_add_)."""
    B = vals.shape[0]
    out = np.zeros((B, n_rows))
    for b in range(B):
        np.add.at(out[b], idx, vals[b])
    return out


class Model:
    """Static per-network data (restates GGASolver.__init__, solver.py:160-495
    and the dense builders :536-1011, :1272-1390, for the batched path)."""

    def __init__(self, net):
        lt = np.asarray(net.link_type, dtype=np.int64)
        nt = np.asarray(net.node_type, dtype=np.int64)
        self.net = net
        self.N, self.L = len(nt), len(lt)
        self.lt = lt
        is_junc = nt == 0
        self.junc = np.flatnonzero(is_junc)
        self.fixed = np.flatnonzero(~is_junc)
        self.Nj = Nj = self.junc.size
        jrow = np.full(self.N, -1, dtype=np.int64)
        jrow[self.junc] = np.arange(Nj)
        n1 = np.asarray(net.link_n1, dtype=np.int64)
        n2 = np.asarray(net.link_n2, dtype=np.int64)
        self.n1, self.n2 = n1, n2
        j1, j2 = jrow[n1], jrow[n2]
        m1, m2 = is_junc[n1], is_junc[n2]
        both = m1 & m2
        self.j1c, self.j2c = np.where(m1, j1, 0), np.where(m2, j2, 0)
        self.m1f, self.m2f = m1.astype(float), m2.astype(float)
        # symmetric slot order fix for >=3 mixed-direction parallel links
        # (solver.py:295-317)
        o1, o2 = j1[both] * Nj + j2[both], j2[both] * Nj + j1[both]
        lo, hi = np.minimum(j1[both], j2[both]), np.maximum(j1[both], j2[both])
        uq, inv, cnt = np.unique(lo * Nj + hi, return_inverse=True, return_counts=True)
        nf = np.zeros(uq.size, dtype=np.int64)
        np.add.at(nf, inv, (j1[both] == lo).astype(np.int64))
        trig = ((cnt >= 3) & (nf != 0) & (nf != cnt))[inv]
        o1 = np.where(trig, lo * Nj + hi, o1)
        o2 = np.where(trig, hi * Nj + lo, o2)
        self.A_idx = np.concatenate([o1, o2, j1[m1] * (Nj + 1), j2[m2] * (Nj + 1)])
        self.lk_both = np.flatnonzero(both)
        self.lk_m1, self.lk_m2 = np.flatnonzero(m1), np.flatnonzero(m2)
        self.f1, self.f2 = j1[m1], j2[m2]
        g1, g2 = (~m1) & m2, (~m2) & m1
        self.lk_g1, self.g1_row, self.g1_src = np.flatnonzero(g1), j2[g1], n1[g1]
        self.lk_g2, self.g2_row, self.g2_src = np.flatnonzero(g2), j1[g2], n2[g2]
        self.lk_f1, self.f1_nodes = np.flatnonzero(~m1), n1[~m1]
        self.lk_f2, self.f2_nodes = np.flatnonzero(~m2), n2[~m2]
        self.fixmask = (~is_junc).astype(float)
        self.el = np.asarray(net.elev_ft, dtype=np.float64)
        self.el_j = self.el[self.junc]
        self.ke_default = np.asarray(net.node_ke, dtype=np.float64)
        meta = net.meta
        form = str(meta.get("headloss", "H-W")).upper()
        if form == "D-W":
            raise NotImplementedError("D-W is epanet-mode only")
        self.hexp = 1.852 if form == "H-W" else 2.0
        self.qexp = float(meta["qexp"])
        self.rqtol = float(meta.get("rqtol", RQTOL))
        self.max_iter_default = int(meta["trials"])
        self.hacc_default = min(max(float(meta["accuracy"]), 1e-5), 1e-1)
        self.htol = float(meta.get("htol", 0.0005))
        self.qtol = float(meta.get("qtol", 0.0001))
        self.checkfreq = int(meta.get("checkfreq", 2))
        self.maxcheck = int(meta.get("maxcheck", 10))
        self.extra_iter = int(meta.get("extra_iter", -1))
        self.r_hw = np.asarray(net.r_hw, dtype=np.float64)
        self.km = np.asarray(net.km_int, dtype=np.float64)
        self.diam = np.asarray(net.diam_ft, dtype=np.float64)
        st = np.asarray(net.init_status)
        setting = np.asarray(net.valve_setting_user, dtype=np.float64)
        d4 = self.diam ** 2 * self.diam ** 2
        self.km_tcv = np.where(st == 2, np.divide(0.02517 * setting, d4,
                                                  out=np.zeros_like(setting),
                                                  where=d4 > 0), self.km)
        self.is_tcv = lt == _TCV
        self.is_pipe = lt <= _PIPE
        self.is_cv = lt == _CVPIPE
        self.closed0 = st == 0
        self.S0 = np.array([{0: CLOSED, 1: OPEN, 2: ACTIVE}[int(s)] for s in st],
                           dtype=np.int8)
        # unit factors (input1.c conversions as restated in solver.py:1291-1305)
        spg = float(meta.get("spgrav", 1.0))
        press = str(meta.get("press_units", "") or "")
        fu = str(meta["flow_units"])
        self.ucf_flow = FLOW_UCF[fu]
        if fu in SI_FLOW:
            self.ucf_head = MperFT
            self.ucf_press = MperFT * spg if (press or "METERS") != "KPA" \
                else KPAperPSI * PSIperFT * spg
        else:
            self.ucf_head = 1.0
            self.ucf_press = PSIperFT * spg
        K0 = setting.copy()
        for k in np.flatnonzero(lt >= _PRV):
            if self.S0[k] != ACTIVE:
                K0[k] = MISSING
            elif lt[k] in (_PRV, _PSV, _PBV):
                K0[k] = K0[k] / self.ucf_press
            elif lt[k] == _FCV:
                K0[k] = K0[k] / self.ucf_flow
        self.K0 = K0
        # pumps (solver.py:950-1011, 1330-1365)
        self.is_pump = lt == _PUMP
        pl = np.asarray(net.pump_link, dtype=np.int64)
        self.n_pumps = pl.size
        L = self.L
        self.p_type = np.full(L, -1)
        self.p_h0, self.p_r, self.p_n = np.zeros(L), np.zeros(L), np.zeros(L)
        self.p_q0, self.p_hmax = np.zeros(L), np.zeros(L)
        if pl.size:
            self.p_type[pl] = np.asarray(net.pump_ptype)
            self.p_h0[pl] = np.asarray(net.pump_h0)
            self.p_r[pl] = np.asarray(net.pump_r)
            self.p_n[pl] = np.asarray(net.pump_n)
            self.p_q0[pl] = np.asarray(net.pump_q0)
            self.p_hmax[pl] = np.asarray(net.pump_hmax)
        pn = self.p_n.copy()
        pn[np.abs(pn - 1.0) < TINY] = 1.0
        self.p_n = pn
        self.p_lin = (pn == 1.0) & self.is_pump
        self.p_pf = self.p_type == 1
        self.p_chp = self.p_type == 0
        self.p_nocurve = self.p_type == 3
        self.p_custom = self.p_type == 2
        sp = K0.copy()
        self.speed = sp
        self.zero_speed = self.is_pump & (sp == 0.0)
        self.pump_live = self.is_pump & (sp > 0.0)
        self.pump_hmax_sm = np.where(self.p_chp, BIG, sp * sp * self.p_hmax)
        self.closed_dense = self.closed0 | self.zero_speed
        self.curves = {}
        if pl.size:
            cq = np.asarray(net.pump_curve_q, dtype=np.float64)
            ch = np.asarray(net.pump_curve_h, dtype=np.float64)
            ptr = np.asarray(net.pump_curve_ptr, dtype=np.int64)
            for j, k in enumerate(pl):
                if self.p_type[k] == 2:
                    self.curves[int(k)] = (cq[ptr[j]:ptr[j + 1]], ch[ptr[j]:ptr[j + 1]])
        # tanks (solver.py:536-568)
        fx = ~is_junc
        tn = np.asarray(net.tank_node, dtype=np.int64)
        is_tank = np.zeros(self.N, dtype=bool)
        is_tank[tn] = True
        thmax, thmin = np.zeros(self.N), np.zeros(self.N)
        tovf = np.zeros(self.N, dtype=bool)
        if tn.size:
            thmax[tn] = np.asarray(net.tank_hmax)
            thmin[tn] = np.asarray(net.tank_hmin)
            tovf[tn] = np.asarray(net.tank_overflow) != 0
        use_n2 = (~fx[n1]) & fx[n2]
        cand = np.where(fx[n1], n1, np.where(fx[n2], n2, -1))
        sel = (cand >= 0) & is_tank[np.where(cand >= 0, cand, 0)]
        k = np.flatnonzero(sel)
        self.tl_k = k
        tank = cand[k]
        self.tl_tank = tank
        self.tl_other = np.where(use_n2[k], n1[k], n2[k])
        self.tl_qsign = np.where(use_n2[k], -1.0, 1.0)
        self.tl_hmax, self.tl_hmin, self.tl_ovf = thmax[tank], thmin[tank], tovf[tank]
        self.tl_is_pump = self.is_pump[k]
        self.tl_pump_in = self.is_pump[k] & (n2[k] == tank)
        self.tl_pump_out = self.is_pump[k] & (n1[k] == tank)
        # PRVs (solver.py:745-832) and PSVs (psvcoeff / psvstatus of the EPANET
        # replica, solver.py:1647-1664, 1736-1765), with a setting, link order
        prv = np.flatnonzero((lt == _PRV) | (lt == _PSV))
        self.pcv = prv[K0[prv] != MISSING]
        self.prv_fixed = np.zeros(L, dtype=bool)
        self.prv_fixed[prv[K0[prv] == MISSING]] = True
        self.pcv_mask = np.zeros(L, dtype=bool)
        self.pcv_mask[self.pcv] = True
        self.prv_psv = lt[self.pcv] == _PSV
        self.prv_n1, self.prv_n2 = n1[self.pcv], n2[self.pcv]
        self.prv_j1, self.prv_j2 = jrow[self.prv_n1], jrow[self.prv_n2]
        # the head an ACTIVE valve holds (PRV n2, PSV n1), its other end, and
        # the sign of the valve flow at the held node
        self.prv_nc = np.where(self.prv_psv, self.prv_n1, self.prv_n2)
        self.prv_jc = np.where(self.prv_psv, self.prv_j1, self.prv_j2)
        self.prv_jo = np.where(self.prv_psv, self.prv_j2, self.prv_j1)
        self.prv_sgn = np.where(self.prv_psv, -1.0, 1.0)
        self.prv_hset = self.el[self.prv_nc] + K0[self.pcv]
        self.prv_km = self.km[self.pcv]
        # FCVs with a flow setting (fcvcoeff / fcvstatus of the EPANET replica,
        # solver.py:1665-1695, 1816-1826, 1875-1877); fixed ones are fixed valves
        fcv = np.flatnonzero(lt == _FCV)
        self.fcv = fcv[K0[fcv] != MISSING]
        self.prv_fixed[fcv[K0[fcv] == MISSING]] = True
        self.fcv_mask = np.zeros(L, dtype=bool)
        self.fcv_mask[self.fcv] = True
        self.fcv_j1, self.fcv_j2 = jrow[n1[self.fcv]], jrow[n2[self.fcv]]
        self.fcv_qs = K0[self.fcv]
        self.fcv_km = self.km[self.fcv]
        self.vmask = self.pcv_mask | self.fcv_mask
        # valvecoeffs visit the valves in link order (hydcoeffs.c:282-330)
        self.vorder = sorted([(int(k), 0, i) for i, k in enumerate(self.pcv)]
                             + [(int(k), 1, j) for j, k in enumerate(self.fcv)])

    # ---------------------------------------------------------------- coeffs
    def pipe_PY(self, q, r):
        """H-W pipe coefficients (solver.py:2176-2201)."""
        sgn = np.where(q < 0, -1.0, 1.0)
        qa = q * sgn
        hg = self.hexp * r * np.maximum(qa, 1e-30) ** (self.hexp - 1.0)
        lin = hg < self.rqtol
        hg = np.where(lin, self.rqtol, hg)
        hl = np.where(lin, hg * qa, hg * qa / self.hexp)
        mp = self.km > 0.0
        hl = np.where(mp, hl + self.km * qa * qa, hl)
        hg = np.where(mp, hg + 2.0 * self.km * qa, hg)
        hl = hl * sgn
        return 1.0 / hg, hl / hg

    def _valve_open(self, q, km):
        """valvecoeff open branch (solver.py:2203-2219, :834-848)."""
        qa = np.abs(q)
        hg = 2.0 * km * qa
        lin = hg < self.rqtol
        hg = np.where(lin, self.rqtol, hg)
        hl = np.where(lin, q * hg, q * hg / 2.0)
        with np.errstate(divide="ignore", invalid="ignore"):
            Pk, Yk = 1.0 / hg, hl / hg
        kp = km > 0.0
        return np.where(kp, Pk, 1.0 / CSMALL), np.where(kp, Yk, q)

    def pump_PY(self, q):
        """Pump coefficients for every curve kind (solver.py:2221-2326)."""
        sgn = np.where(q < 0, -1.0, 1.0)
        qa = q * sgn
        spc = np.maximum(self.speed, 1e-12)
        h0e = spc * spc * self.p_h0
        re = self.p_r * spc ** (2.0 - self.p_n)
        with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
            qa_c = np.maximum(qa, 1e-30)
            raw = -re / qa_c / qa_c
            big, sml = raw > CBIG, raw < self.rqtol
            hg_c = np.where(big, CBIG, np.where(sml, self.rqtol, raw))
            hl_c = np.where(big | sml, -hg_c * q, re / (sgn * qa_c))
            qz = qa == 0.0
            nm1 = self.p_n - 1.0
            pw0 = np.where(nm1 > 0.0, 0.0, np.where((nm1 < 0.0) & self.p_pf, np.inf, 1.0))
            qpf = np.where(qz, 1.0, qa)
            raw = self.p_n * re * np.where(qz, pw0, qpf ** nm1)
            sml = raw < self.rqtol
            hg_p = np.where(sml, self.rqtol, raw)
            hl_p = np.where(sml, h0e + hg_p * q,
                            h0e + hg_p * q / np.maximum(self.p_n, 1e-30))
            hg_p = np.where(self.p_lin, re, hg_p)
            hl_p = np.where(self.p_lin, h0e + re * q, hl_p)
            hg = np.where(self.p_chp, hg_c, hg_p)
            hl = np.where(self.p_chp, hl_c, hl_p)
            for k, (cx, cy) in self.curves.items():
                s = max(self.speed[k], 1e-12)
                qq = (np.abs(q[:, k]) / s) * self.ucf_flow
                idx = np.searchsorted(cx, qq, side="left")
                k2 = np.minimum(np.maximum(idx, 1), cx.size - 1)
                k1 = k2 - 1
                rc = (cy[k2] - cy[k1]) / (cx[k2] - cx[k1])
                h0c = cy[k1] - rc * cx[k1]
                h0c = h0c / self.ucf_head
                rc = rc * self.ucf_flow / self.ucf_head
                hg[:, k] = (-rc) * s
                hl[:, k] = (-h0c) * (s * s) + hg[:, k] * q[:, k]
            P, Y = 1.0 / hg, hl / hg
        P = np.where(self.p_nocurve, 1.0 / CSMALL, P)
        Y = np.where(self.p_nocurve, q, Y)
        return P, Y

    def with_pumps(self, speed=None, h0=None, r=None):
        """A copy of the model at a call's pump parameters ([L] rows, read at
        pump links): the speed / pump_h0 / pump_r of implicit_solve
        (autodiff.py:99-120 _resolve_pump_args).  Speed also sets the
        zero-speed closed branch and the pumpstatus shut-off head
        (solver.py:665-679)."""
        m = copy.copy(self)
        if speed is not None:
            sp = np.where(self.is_pump, np.asarray(speed, dtype=np.float64), self.speed)
            m.speed = sp
            m.zero_speed = self.is_pump & (sp == 0.0)
            m.pump_live = self.is_pump & (sp > 0.0)
            m.pump_hmax_sm = np.where(self.p_chp, BIG, sp * sp * self.p_hmax)
            m.closed_dense = self.closed0 | m.zero_speed
        if h0 is not None:
            m.p_h0 = np.where(self.is_pump, np.asarray(h0, dtype=np.float64), self.p_h0)
        if r is not None:
            m.p_r = np.where(self.is_pump, np.asarray(r, dtype=np.float64), self.p_r)
        return m

    def pump_dtheta(self, q, S):
        """d hloss / d(speed, H0, R) of every pump at flows q [B,L] with the
        statuses S frozen (autodiff.py:122-218 _pump_coeffs_np,
        hydcoeffs.c:673-791); three [B,L] arrays, zero off pumps and on the
        closed / zero-speed / NOCURVE / clamped constant-HP branches."""
        B = q.shape[0]
        dw, dh0, dR = np.zeros((B, self.L)), np.zeros((B, self.L)), np.zeros((B, self.L))
        for k in np.flatnonzero(self.is_pump):
            w = float(self.speed[k])
            t = int(self.p_type[k])
            for b in range(B):
                if S is not None and S[b, k] <= CLOSED or w == 0.0 or t == 3:
                    continue
                qk = float(q[b, k])
                qa = abs(qk)
                if t == 2:   # frozen curve segment: hloss = w^2 H0c + w Rc q
                    cx, cy = self.curves[int(k)]
                    qq = (qa / w) * self.ucf_flow
                    i2 = min(max(int(np.searchsorted(cx, qq, side="left")), 1), cx.size - 1)
                    i1 = i2 - 1
                    rc = (cy[i2] - cy[i1]) / (cx[i2] - cx[i1])
                    h0c = (cy[i1] - rc * cx[i1]) / self.ucf_head
                    rc = rc * self.ucf_flow / self.ucf_head
                    dw[b, k] = 2.0 * w * (-h0c) + (-rc) * qk
                    continue
                n, H0, R = float(self.p_n[k]), float(self.p_h0[k]), float(self.p_r[k])
                if t == 0:   # constant HP: hloss = r / q, r = R w^(2-n)
                    hgr = -(R * w ** (2.0 - n)) / qa / qa if qa > 0.0 else np.inf
                    if self.rqtol <= hgr <= CBIG:
                        dw[b, k] = (2.0 - n) * R * w ** (1.0 - n) / qk
                        dR[b, k] = w ** (2.0 - n) / qk
                    continue
                dh0[b, k] = w * w
                if n == 1.0:  # linear curve: hloss = w^2 H0 + R w q
                    dw[b, k] = 2.0 * w * H0 + R * qk
                    dR[b, k] = w * qk
                    continue
                pw = qa ** (n - 1.0) if qa > 0.0 else (0.0 if n > 1.0 else np.inf)
                if n * (R * w ** (2.0 - n)) * pw < self.rqtol:   # RQtol clamp
                    dw[b, k] = 2.0 * w * H0
                    continue
                dw[b, k] = 2.0 * w * H0 + (2.0 - n) * R * w ** (1.0 - n) * pw * qk
                dR[b, k] = w ** (2.0 - n) * pw * qk
        return dw, dh0, dR

    def chp_clamp(self, q, S):
        """[B,L] mask of open constant-HP pumps on their CBIG / RQtol clamp
        branch (hydcoeffs.c:748-757): there hloss = -hgrad q, so the exact
        d hloss / dq of the CPU adjoint is -hgrad (autodiff.py:186-193) where
        the GGA matrix assembles +hgrad."""
        B = q.shape[0]
        out = np.zeros((B, self.L), dtype=bool)
        for k in np.flatnonzero(self.is_pump & self.p_chp):
            w = float(self.speed[k])
            if w == 0.0:
                continue
            re = self.p_r[k] * max(w, 1e-12) ** (2.0 - self.p_n[k])
            for b in range(B):
                if S is not None and S[b, k] <= CLOSED:
                    continue
                qa = max(abs(float(q[b, k])), 1e-30)
                raw = -re / qa / qa
                out[b, k] = raw > CBIG or raw < self.rqtol
        return out

    def emitter(self, e, ke):
        """Emitter head loss and gradient (solver.py:2368-2377)."""
        kea = np.maximum(ke, CSMALL)
        hg = self.qexp * kea * np.maximum(np.abs(e), 1e-30) ** (self.qexp - 1.0)
        lin = hg < self.rqtol
        hg = np.where(lin, self.rqtol, hg)
        hl = np.where(lin, hg * e, hg * e / self.qexp)
        return hl, hg

    def headloss_PY(self, q, r, S):
        """Link P, Y before the valve stage (solver.py:2923-2956)."""
        P, Y = self.pipe_PY(q, r)
        Pt, Yt = self._valve_open(q, self.km_tcv)
        P, Y = np.where(self.is_tcv, Pt, P), np.where(self.is_tcv, Yt, Y)
        if self.n_pumps:
            Pp, Yp = self.pump_PY(q)
            P, Y = np.where(self.is_pump, Pp, P), np.where(self.is_pump, Yp, Y)
        if self.prv_fixed.any():
            Pv, Yv = self._valve_open(q, self.km)
            P, Y = np.where(self.prv_fixed, Pv, P), np.where(self.prv_fixed, Yv, Y)
        closed = ((S <= CLOSED) | self.zero_speed) if S is not None else self.closed_dense
        if self.vmask.any():
            closed = closed & ~self.vmask
        P = np.where(closed, 1.0 / CBIG, P)
        Y = np.where(closed, q, Y)
        if self.vmask.any():
            P = np.where(self.vmask, 0.0, P)
            Y = np.where(self.vmask, 0.0, Y)
        return P, Y, closed

    def _fcv_coeffs(self, j, P, Y, F, A, Xflow, q, S):
        """One FCV in the valve pass (fcvcoeff, solver.py:1665-1695): ACTIVE
        cuts the network (an outflow qset at n1, an inflow at n2, P = 1/CBIG,
        Y = q - qset); otherwise the open / closed valve coefficients."""
        Nj = self.Nj
        k, j1, j2, qs = self.fcv[j], self.fcv_j1[j], self.fcv_j2[j], self.fcv_qs[j]
        qk, sk = q[:, k], S[:, k]
        act = sk == ACTIVE
        cl = sk <= CLOSED
        km = self.fcv_km[j]
        if km > 0.0:
            hg = 2.0 * km * np.abs(qk)
            lin = hg < self.rqtol
            hg = np.where(lin, self.rqtol, hg)
            hl = np.where(lin, qk * hg, qk * hg / 2.0)
            po, yo = 1.0 / hg, hl / hg
        else:
            po, yo = np.full_like(qk, 1.0 / CSMALL), qk
        pv, yv = np.where(cl, 1.0 / CBIG, po), np.where(cl, qk, yo)
        pk = np.where(act, 1.0 / CBIG, pv)
        yk = np.where(act, qk - qs, yv)
        Xflow[:, j1] -= qs * act
        Xflow[:, j2] += qs * act
        F[:, j1] += np.where(act, -qs, yv - qk)
        F[:, j2] += np.where(act, qs, -(yv - qk))
        if A is not None:
            for slot, v in ((j1 * Nj + j2, -pk), (j2 * Nj + j1, -pk),
                            (j1 * Nj + j1, pk), (j2 * Nj + j2, pk)):
                A[:, slot] += v
        P[:, k] = pk
        Y[:, k] = yk

    def prv_coeffs(self, P, Y, F, A, Xflow, q, S):
        """Batched valve coefficients after nodecoeffs, in valve (link) order:
        PRVs as solver.py:850-912, FCVs as `_fcv_coeffs`.  A is the dense
        [B,Nj*Nj] matrix (or None)."""
        Nj = self.Nj
        for _, kind, i in self.vorder:
            if kind == 1:
                self._fcv_coeffs(i, P, Y, F, A, Xflow, q, S)
                continue
            k = self.pcv[i]
            j1, j2 = self.prv_j1[i], self.prv_j2[i]
            qk, sk = q[:, k], S[:, k]
            act, cl = sk == ACTIVE, sk <= CLOSED
            km = self.prv_km[i]
            if km > 0.0:
                qa = np.abs(qk)
                hg = 2.0 * km * qa
                lin = hg < self.rqtol
                hg = np.where(lin, self.rqtol, hg)
                hl = np.where(lin, qk * hg, qk * hg / 2.0)
                po, yo = 1.0 / hg, hl / hg
            else:
                po, yo = np.full_like(qk, 1.0 / CSMALL), qk
            pna = np.where(cl, 1.0 / CBIG, po) * (~act)
            yna = np.where(cl, qk, yo)
            jc, jo, sg = self.prv_jc[i], self.prv_jo[i], self.prv_sgn[i]
            xfc = Xflow[:, jc]
            dy = (yna - qk) * (~act)
            if A is not None:
                for slot, v in ((j1 * Nj + j2, -pna), (j2 * Nj + j1, -pna),
                                (j1 * Nj + j1, pna), (j2 * Nj + j2, pna),
                                (jc * Nj + jc, CBIG * act)):
                    A[:, slot] += v
            F[:, j1] += dy
            F[:, j2] -= dy
            F[:, jo] += np.where(act & (sg * xfc < 0.0), xfc, 0.0)
            F[:, jc] += self.prv_hset[i] * CBIG * act
            P[:, k] = pna
            Y[:, k] = np.where(act, qk + sg * xfc, yna)
        return P, Y, F, A

    # ---------------------------------------------------------- status
    def _cv_closed(self, s_open, dh, q):
        big = np.abs(dh) > self.htol
        cb = (dh < -self.htol) | (q < -self.qtol)
        cs = (q < -self.qtol) if s_open else np.ones_like(cb)
        return np.where(big, cb, cs)

    def link_status(self, S, H, q):
        """linkstatus batch (solver.py:697-739)."""
        st0 = S
        s = np.where((st0 == XHEAD) | (st0 == TEMPCLOSED), OPEN, st0).astype(np.int8)
        dh = H[:, self.n1] - H[:, self.n2]
        if self.is_cv.any():
            big = np.abs(dh) > self.htol
            rev = q < -self.qtol
            nb = np.where((dh < -self.htol) | rev, CLOSED, OPEN)
            ns = np.where(rev, CLOSED, s)
            s = np.where(self.is_cv, np.where(big, nb, ns), s).astype(np.int8)
        if self.n_pumps:
            xh = np.where(-dh > self.pump_hmax_sm + self.htol, XHEAD, OPEN)
            s = np.where(self.pump_live & (s >= OPEN), xh, s).astype(np.int8)
        if self.fcv.size:   # fcvstatus from the status before the reopening
            kf = self.fcv
            qk, s0 = q[:, kf], st0[:, kf]
            rev = (dh[:, kf] < -self.htol) | (qk < -self.qtol)
            s[:, kf] = np.where(rev, XFCV, np.where((s0 == XFCV) & (qk >= self.fcv_qs),
                                                    ACTIVE, s0))
        k = self.tl_k
        if k.size:
            live = s[:, k] > CLOSED
            ht = H[:, self.tl_tank]
            dht = ht - H[:, self.tl_other]
            qk = q[:, k] * self.tl_qsign
            full = (ht >= self.tl_hmax - self.htol) & (~self.tl_ovf)
            empty = ht <= self.tl_hmin + self.htol
            cf = np.where(self.tl_is_pump, self.tl_pump_in, self._cv_closed(True, dht, qk))
            ce = np.where(self.tl_is_pump, self.tl_pump_out, ~self._cv_closed(False, dht, qk))
            hit = live & ((full & cf) | (empty & ce))
            s[:, k] = np.where(hit, TEMPCLOSED, s[:, k])
        return s, (s != st0).any(axis=1)

    def prv_status(self, S, H, q):
        """prvstatus batch (solver.py:914-947)."""
        k = self.pcv
        h1, h2 = H[:, self.prv_n1], H[:, self.prv_n2]
        qk, sk = q[:, k], S[:, k]
        hs, ht, qt = self.prv_hset, self.htol, self.qtol
        hml = self.prv_km * (qk * qk)
        neg = qk < -qt
        c_act = np.where(neg, CLOSED, np.where(h1 - hml < hs - ht, OPEN, ACTIVE))
        c_open = np.where(neg, CLOSED, np.where(h2 >= hs + ht, ACTIVE, OPEN))
        c_cl = np.where((h1 >= hs + ht) & (h2 < hs - ht), ACTIVE,
                        np.where((h1 < hs - ht) & (h1 > h2 + ht), OPEN, CLOSED))
        c_xp = np.where(neg, CLOSED, sk)
        if self.prv_psv.any():   # psvstatus (solver.py:1736-1765)
            v = self.prv_psv
            c_act = np.where(v, np.where(neg, CLOSED, np.where(h2 + hml > hs + ht, OPEN, ACTIVE)),
                             c_act)
            c_open = np.where(v, np.where(neg, CLOSED, np.where(h1 < hs - ht, ACTIVE, OPEN)),
                              c_open)
            c_cl = np.where(v, np.where((h2 > hs + ht) & (h1 > h2 + ht), OPEN,
                                        np.where((h1 >= hs + ht) & (h1 > h2 + ht), ACTIVE, CLOSED)),
                            c_cl)
        new = np.where(sk == ACTIVE, c_act, np.where(sk == OPEN, c_open,
                       np.where(sk == CLOSED, c_cl, np.where(sk == XPRESSURE, c_xp, sk))))
        new = new.astype(np.int8)
        out = S.copy()
        out[:, k] = new
        return out, (new != sk).any(axis=1)

    # ---------------------------------------------------------- forward
    def init_flow(self):
        """solver.py:2163-2174."""
        q = PI * self.diam ** 2 / 4.0
        if self.n_pumps:
            q = np.where(self.is_pump, self.K0 * self.p_q0, q)
        return np.where(self.closed0, QZERO, q)

    def _assemble(self, P, Y, q, H, e, ke, d, S):
        B, Nj = q.shape[0], self.Nj
        pl = (P != 0.0).astype(float)
        Pm, Ym, qm = P * pl, Y * pl, q * pl
        Xf = _scatter(Nj, self.f1, -qm[:, self.lk_m1])
        Xf = Xf + 0.0
        for b in range(B):
            np.add.at(Xf[b], self.f2, qm[b, self.lk_m2])
        vals = np.concatenate([-Pm[:, self.lk_both], -Pm[:, self.lk_both],
                               Pm[:, self.lk_m1], Pm[:, self.lk_m2]], axis=1)
        A = _scatter(Nj * Nj, self.A_idx, vals)
        F = _scatter(Nj, self.f1, Ym[:, self.lk_m1])
        for b in range(B):
            np.add.at(F[b], self.f2, -Ym[b, self.lk_m2])
            if self.lk_g1.size:
                np.add.at(F[b], self.g1_row, Pm[b, self.lk_g1] * H[b, self.g1_src])
            if self.lk_g2.size:
                np.add.at(F[b], self.g2_row, Pm[b, self.lk_g2] * H[b, self.g2_src])
        hle, hge = self.emitter(e, ke)
        em = (ke > 0.0).astype(float)
        diag = np.arange(Nj) * (Nj + 1)
        A[:, diag] = A[:, diag] + em / hge
        F = F + em * (hle + self.el_j) / hge
        Xf = Xf - em * e
        Xf = Xf - d
        F = F + Xf
        if self.vmask.any():
            P, Y, F, A = self.prv_coeffs(P.copy(), Y.copy(), F, A, Xf, q, S)
        return P, Y, F, A.reshape(B, Nj, Nj), hle, hge, em

    @staticmethod
    def _chol_solve(A, F, n_refine=2):
        B = A.shape[0]
        x = np.empty_like(F)
        for b in range(B):
            c = sla.cho_factor(A[b], lower=True)
            xb = sla.cho_solve(c, F[b])
            for _ in range(n_refine):
                xb = xb + sla.cho_solve(c, F[b] - (A[b] * xb[None, :]).sum(-1))
            x[b] = xb
        return x

    def solve(self, d, rh, ke=None, r=None, accuracy=None, max_iter=None,
              status_machine=False, q0=None, e0=None, S0=None):
        """Batched steady solve (restates solver.py:2703-3212); q0 [B or 1, L]
        and e0 [B or 1, N] are the warm start of solver.py:2876-2887; S0
        [B or 1, L] the initial statuses (run_gga(status0=), the frame-to-frame
        carry of dgga/eps.py:366-373)."""
        d = np.atleast_2d(np.asarray(d, dtype=np.float64))
        B = d.shape[0]
        rh = np.broadcast_to(np.atleast_2d(rh), (B, self.N))
        ke = self.ke_default if ke is None else np.asarray(ke, dtype=np.float64)
        ke = np.broadcast_to(np.atleast_2d(ke), (B, self.N))
        r = self.r_hw if r is None else np.asarray(r, dtype=np.float64)
        r = np.broadcast_to(r, (B, self.L))
        ke_j, d_j = ke[:, self.junc], d[:, self.junc]
        has_em = ke_j > 0.0
        max_iter = self.max_iter_default if max_iter is None else int(max_iter)
        hacc = self.hacc_default if accuracy is None else float(accuracy)
        q0 = self.init_flow() if q0 is None else np.asarray(q0, dtype=np.float64)
        q = np.broadcast_to(q0, (B, self.L)).copy()
        if e0 is None:
            e = np.where(has_em, 1.0, 0.0)
        else:
            e0 = np.broadcast_to(np.atleast_2d(np.asarray(e0, dtype=np.float64)), (B, self.N))
            e = np.where(has_em, e0[:, self.junc], 0.0)
        H = np.array(rh, dtype=np.float64)
        H[:, self.junc] = 0.0
        if np.isnan(H[:, self.fixed]).any():
            raise ValueError("res_head_ft is nan at a reservoir/tank node")
        active = np.ones(B, dtype=bool)
        iters = np.zeros(B, dtype=np.int64)
        relerr_out = np.zeros(B)
        sm = bool(status_machine)
        maxtrials = max_iter
        S = nextcheck = None
        if sm:
            S = np.broadcast_to(self.S0 if S0 is None else S0, (B, self.L)).copy()
            maxtrials = max_iter + (self.extra_iter if self.extra_iter > 0 else 0)
            nextcheck = np.full(B, self.checkfreq, dtype=np.int64)
        elif self.vmask.any() or self.is_cv.any():
            raise NotImplementedError("PRV/FCV/CV networks need status_machine=True")
        for it in range(1, maxtrials + 1):
            P, Y, _ = self.headloss_PY(q, r, S)
            P, Y, F, A, hle, hge, em = self._assemble(P, Y, q, H, e, ke_j, d_j, S)
            Hj = self._chol_solve(A, F)
            H[:, self.junc] = np.where(active[:, None], Hj, H[:, self.junc])
            dh = H[:, self.n1] - H[:, self.n2]
            dq = Y - P * dh
            if self.n_pumps:
                dq = np.where(self.p_chp & (dq > q), q / 2.0, dq)
            qn = q - dq
            dqe = (hle - (H[:, self.junc] - self.el_j)) / hge
            en = e - em * dqe
            dqs = np.abs(dq).sum(1) + (em * np.abs(dqe)).sum(1)
            qs = np.abs(qn).sum(1) + (em * np.abs(en)).sum(1)
            relerr = np.where(qs > hacc, dqs / qs, dqs)
            q = np.where(active[:, None], qn, q)
            e = np.where(active[:, None], en, e)
            iters = np.where(active, it, iters)
            relerr_out = np.where(active, relerr, relerr_out)
            if not sm:
                active = active & (relerr > hacc)
                if not active.any():
                    break
                continue
            vchg = None
            if self.pcv.size:
                Sv, vc = self.prv_status(S, H, q)
                S = np.where(active[:, None], Sv, S)
                vchg = vc & active
            conv = relerr <= hacc
            br_conv = active & conv & (it <= max_iter)
            br_per = active & ~conv & (it <= self.maxcheck) & (nextcheck == it)
            run = br_conv | br_per
            Sn, chg = self.link_status(S, H, q)
            S = np.where(run[:, None], Sn, S)
            sc = chg & br_conv
            if vchg is not None:
                sc = sc | (vchg & br_conv)
            nextcheck = np.where(br_conv & sc, it + self.checkfreq, nextcheck)
            nextcheck = np.where(br_per, nextcheck + self.checkfreq, nextcheck)
            done = active & conv & ((it > max_iter) | ~sc)
            active = active & ~done
            if not active.any():
                break
        iters = np.where(active, maxtrials + 1, iters)
        emit = np.zeros((B, self.N))
        emit[:, self.junc] = e * has_em
        out = dict(head_ft=H, flow_cfs=q, emitter_cfs=emit, iters=iters,
                   relerr=relerr_out, converged=~active)
        if sm:
            out["status"] = S
        return out

    # ---------------------------------------------------------- polish/adjoint
    def adj_coeffs(self, q, e, ke, r, S):
        """Coefficients at the current state (autodiff.py:786-875)."""
        P, Y, closed = self.headloss_PY(q, r, S)
        act = None
        if self.vmask.any():
            B = q.shape[0]
            Yd = np.zeros_like(q)
            P, Y2, _, _ = self.prv_coeffs(P.copy(), Yd, np.zeros((B, self.Nj)), None,
                                          np.zeros((B, self.Nj)), q, S)
            Y = Y.copy()
            Y[:, self.vmask] = Y2[:, self.vmask]
            if self.pcv.size:
                act = S[:, self.pcv] == ACTIVE
        _, hge = self.emitter(e, ke)
        em = (ke > 0.0).astype(float)
        emh = em / hge
        sgn = np.where(q < 0, -1.0, 1.0)
        qa = q * sgn
        hgr = self.hexp * r * np.maximum(qa, 1e-30) ** (self.hexp - 1.0)
        dr = np.where(self.is_pipe & ~closed & (hgr >= self.rqtol), qa ** self.hexp * sgn, 0.0)
        ea = np.abs(e)
        hraw = self.qexp * np.maximum(ke, CSMALL) * np.maximum(ea, 1e-30) ** (self.qexp - 1.0)
        dke = np.where((hraw < self.rqtol) | (ke < CSMALL), 0.0,
                       np.maximum(ea, 1e-30) ** (self.qexp - 1.0) * e)
        return P, Y, emh, hge, em, dr, dke, act

    def matvec(self, P, emh, act, x):
        """A x for the reduced matrix (autodiff.py:878-895)."""
        t = P * (x[:, self.j1c] * self.m1f - x[:, self.j2c] * self.m2f)
        out = _scatter(self.Nj, self.f1, t[:, self.lk_m1])
        for b in range(x.shape[0]):
            np.add.at(out[b], self.f2, -t[b, self.lk_m2])
        out = out + emh * x
        if act is not None:
            for b in range(x.shape[0]):
                np.add.at(out[b], self.prv_jc, x[b, self.prv_jc] * act[b] * CBIG)
        return out

    def factor(self, P, emh, act, lu=False):
        """Assemble the reduced matrix at the current state and factor it
        (autodiff.py:928-962); lu: an LU factor, for the indefinite matrix of
        the exact Jacobian with clamped constant-HP pumps."""
        B, Nj = P.shape[0], self.Nj
        vals = np.concatenate([-P[:, self.lk_both], -P[:, self.lk_both],
                               P[:, self.lk_m1], P[:, self.lk_m2]], axis=1)
        A = _scatter(Nj * Nj, self.A_idx, vals)
        diag = np.arange(Nj) * (Nj + 1)
        A[:, diag] += emh
        if act is not None and act.any():
            for b in range(B):
                np.add.at(A[b], self.prv_jc * (Nj + 1), CBIG * act[b])
        A = A.reshape(B, Nj, Nj)
        if lu:
            return [("lu", sla.lu_factor(A[b])) for b in range(B)]
        return [sla.cho_factor(A[b], lower=True) for b in range(B)]

    @staticmethod
    def _fsolve(kf, rhs):
        return np.stack([sla.lu_solve(kf[b][1], rhs[b]) if isinstance(kf[b][0], str)
                         else sla.cho_solve(kf[b], rhs[b]) for b in range(rhs.shape[0])])

    def _solveA(self, kf, P, emh, act, rhs, n_ref=2):
        x = self._fsolve(kf, rhs)
        for _ in range(n_ref):
            x = x + self._fsolve(kf, rhs - self.matvec(P, emh, act, x))
        return x

    def primal_solve(self, kf, P, emh, act, rhs, r_prv):
        """Reduced Newton system with ACTIVE-PRV rows (autodiff.py:965-1029)."""
        if act is None or not act.any():
            return self._solveA(kf, P, emh, act, rhs)
        B, p = rhs.shape[0], act.shape[1]
        j1, j2 = self.prv_jo, self.prv_jc     # other end, held node
        actf = act.astype(float)
        rp = rhs.copy()
        for b in range(B):
            np.add.at(rp[b], j1, np.where(act[b], rhs[b, j2], 0.0))
        rp[:, j2] = np.where(act, -r_prv, rhs[:, j2])
        x0 = self._solveA(kf, P, emh, act, rp)
        cols = []
        for u in list(j2) + list(j1):
            eb = np.zeros_like(rhs)
            eb[:, u] = 1.0
            cols.append(self._solveA(kf, P, emh, act, eb))
        Sm = np.stack(cols, axis=-1)
        R2 = Sm[:, j2, :]
        eye2 = np.tile(np.eye(p), (1, 2))[None]
        C = np.concatenate([R2, eye2 - CBIG * R2], axis=1)
        a2 = np.concatenate([actf, actf], axis=1)
        Ce = C * a2[:, :, None] + np.stack([np.diag(1.0 - v) for v in a2])

        def wood(x, rr):
            top = (x[:, j2] - rr[:, j2]) * actf
            bot = (rr[:, j2] - CBIG * x[:, j2]) * actf
            y = np.linalg.solve(Ce, np.concatenate([top, bot], 1)[..., None])[..., 0]
            return x - np.einsum("bnp,bp->bn", Sm, y)

        dH = wood(x0, rp)
        for _ in range(2):
            base = self.matvec(P, emh, act, dH)
            row1 = base[:, j1] + base[:, j2] - CBIG * dH[:, j2]
            res = rp - base
            res[:, j1] = np.where(act, rp[:, j1] - row1, res[:, j1])
            res[:, j2] = np.where(act, rp[:, j2] - dH[:, j2], res[:, j2])
            dH = dH + wood(self._solveA(kf, P, emh, act, res), res)
        return dH

    def residuals(self, q, e, H, d, ke, P, Y, em, act):
        """autodiff.py:1032-1050."""
        with np.errstate(divide="ignore", invalid="ignore"):
            hl = np.where(P != 0.0, Y / P, 0.0)
        r_l = hl - (H[:, self.n1] - H[:, self.n2])
        r_prv = None
        if act is not None:
            r_prv = (H[:, self.prv_nc] - self.prv_hset) * act
        hle, _ = self.emitter(e, ke)
        r_e = hle - (H[:, self.junc] - self.el_j)
        m = _scatter(self.Nj, self.f2, q[:, self.lk_m2])
        for b in range(q.shape[0]):
            np.add.at(m[b], self.f1, -q[b, self.lk_m1])
        m = m - em * e - d
        return r_l, r_prv, r_e, m

    def polish(self, q, e, H, d, ke, r, S, steps):
        """Reduced Newton polish + terminal factor (autodiff.py:1053-1104)."""
        q, e, H = q.copy(), e.copy(), H.copy()
        for _ in range(steps):
            P, Y, emh, hge, em, dr, dke, act = self.adj_coeffs(q, e, ke, r, S)
            kf = self.factor(P, emh, act)
            r_l, r_prv, r_e, m = self.residuals(q, e, H, d, ke, P, Y, em, act)
            Pr = P * r_l
            bt = _scatter(self.Nj, self.f2, Pr[:, self.lk_m2])
            for b in range(q.shape[0]):
                np.add.at(bt[b], self.f1, -Pr[b, self.lk_m1])
            rhs = m - bt + emh * r_e
            dH = self.primal_solve(kf, P, emh, act, rhs, r_prv)
            dq = -P * (r_l + (dH[:, self.j2c] * self.m2f - dH[:, self.j1c] * self.m1f))
            if act is not None and act.any():
                base = self.matvec(P, emh, act, dH)
                ab2 = base[:, self.prv_jc] - CBIG * dH[:, self.prv_jc] * act
                dqp = self.prv_sgn * (rhs[:, self.prv_jc] - ab2)
                dq[:, self.pcv] = np.where(act, dqp, dq[:, self.pcv])
            de = em * (-r_e + dH) / hge
            q = q + dq
            e = e + de
            H[:, self.junc] = H[:, self.junc] + dH
        P, Y, emh, hge, em, dr, dke, act = self.adj_coeffs(q, e, ke, r, S)
        kf = self.factor(P, emh, act)
        return q, e, H, kf

    def node_solve(self, kf, P, emh, act, r, gQp):
        """Adjoint node system with constraint rows (autodiff.py:1107-1154)."""
        if act is None or not act.any():
            return self._solveA(kf, P, emh, act, r)
        B, p = r.shape[0], act.shape[1]
        j1, j2 = self.prv_jo, self.prv_jc     # other end, held node
        actf = act.astype(float)
        r2 = r.copy()
        r2[:, j2] = np.where(act, self.prv_sgn * gQp, r[:, j2])
        x0 = self._solveA(kf, P, emh, act, r2)
        cols = []
        for u in j2:
            eb = np.zeros_like(r)
            eb[:, u] = 1.0
            cols.append(self._solveA(kf, P, emh, act, eb))
        Sm = np.stack(cols, axis=-1)
        Cw = Sm[:, j2, :] - Sm[:, j1, :]
        Ce = Cw * (actf[:, :, None] * actf[:, None, :]) + np.stack([np.diag(1.0 - v) for v in actf])

        def wood(x, rr):
            w = (x[:, j2] - x[:, j1] - rr[:, j2]) * actf
            y = np.linalg.solve(Ce, w[..., None])[..., 0]
            return x - np.einsum("bnp,bp->bn", Sm, y)

        lam = wood(x0, r2)
        for _ in range(2):
            res = r2 - self.matvec(P, emh, act, lam)
            con = r2[:, j2] - (lam[:, j2] - lam[:, j1])
            res[:, j2] = np.where(act, con, res[:, j2])
            lam = lam + wood(self._solveA(kf, P, emh, act, res), res)
        return lam

    def adjoint(self, q, e, ke, r, S, kf, gH, gQ, gE, pumps=False):
        """Reduced adjoint (autodiff.py:1246-1312); gradients stay [B,*].
        pumps: also the pump-theta gradients (d speed, d H0, d R) [B,L]."""
        B = q.shape[0]
        P, _, emh, hge, em, dr, dke, act = self.adj_coeffs(q, e, ke, r, S)
        clamp = self.chp_clamp(q, S)
        if clamp.any():   # exact Jacobian: -hgrad on the clamp branch
            P = np.where(clamp, -P, P)
            kf = self.factor(P, emh, act, lu=True)
        gHj, gEj = gH[:, self.junc], gE[:, self.junc]
        PgQ = P * gQ
        rr = _scatter(self.Nj, self.f2, PgQ[:, self.lk_m2])
        for b in range(B):
            np.add.at(rr[b], self.f1, -PgQ[b, self.lk_m1])
        rr = rr - emh * gEj - gHj
        gQp = gQ[:, self.pcv] if act is not None else None
        lam = self.node_solve(kf, P, emh, act, rr, gQp)
        lam_l = P * (gQ - (lam[:, self.j2c] * self.m2f - lam[:, self.j1c] * self.m1f))
        lam_e = em * (gEj + lam) / hge
        gd = np.zeros((B, self.N))
        gd[:, self.junc] = lam
        gke = np.zeros((B, self.N))
        gke[:, self.junc] = -(lam_e * dke)
        grh = np.zeros((B, self.N))
        for b in range(B):
            np.add.at(grh[b], self.f1_nodes, lam_l[b, self.lk_f1])
            np.add.at(grh[b], self.f2_nodes, -lam_l[b, self.lk_f2])
        grh = grh + gH * self.fixmask
        gr = -(lam_l * dr)
        if pumps:   # pump theta: -lam_l d hloss / d theta (autodiff.py:736-741)
            return (gd, grh, gke, gr) + tuple(-(lam_l * x) for x in self.pump_dtheta(q, S))
        return gd, grh, gke, gr

    def implicit(self, d, rh, ke=None, r=None, accuracy=1e-12, max_iter=200,
                 polish_steps=3, status_machine=True, q0=None, e0=None, S0=None):
        """Forward + polish; returns (out, state) where state feeds adjoint()."""
        d = np.atleast_2d(np.asarray(d, dtype=np.float64))
        B = d.shape[0]
        ke = self.ke_default if ke is None else np.asarray(ke, dtype=np.float64)
        ke = np.broadcast_to(np.atleast_2d(ke), (B, self.N))
        r = self.r_hw if r is None else np.asarray(r, dtype=np.float64)
        r = np.broadcast_to(r, (B, self.L))
        out = self.solve(d, rh, ke=ke, r=r, accuracy=accuracy, max_iter=max_iter,
                         status_machine=status_machine, q0=q0, e0=e0, S0=S0)
        if not out["converged"].all():
            raise RuntimeError("unconverged scenarios %s" %
                               np.flatnonzero(~out["converged"]).tolist())
        S = out.get("status")
        e = out["emitter_cfs"][:, self.junc]
        ke_j, d_j = ke[:, self.junc], d[:, self.junc]
        q, e, H, kf = self.polish(out["flow_cfs"], e, out["head_ft"], d_j, ke_j,
                                  r, S, polish_steps)
        em = (ke_j > 0.0).astype(float)
        emit = np.zeros((B, self.N))
        emit[:, self.junc] = e * em
        state = dict(q=q, e=e, ke=ke_j, r=r, S=S, kf=kf)
        return dict(head_ft=H, flow_cfs=q, emitter_cfs=emit, iters=out["iters"],
                    status=S), state

    def backward(self, state, gH, gQ, gE, pumps=False):
        return self.adjoint(state["q"], state["e"], state["ke"], state["r"],
                            state["S"], state["kf"], gH, gQ, gE, pumps=pumps)
