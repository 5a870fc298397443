"""GGASolver with the B200 route: the reference's batched dense/CSR GGA
(`dgga.solver.GGASolver`, dgga/solver.py:160-3212) behind the same
constructor and `solve()` signature, with the per-iteration body and the
linear solver replaced by one fused sm_100a kernel launch
(`linear_solver="sm100"`, `assemble="csr"`).

Host side only: this module validates the network with the reference's
admission rules and error classes, derives the per-link tables the reference
builds in `__init__` (dgga/solver.py:239-1011, 1272-1390), hands them to the
C ABI (`wds_plan`) and calls `wds_forward` on the current torch stream.  There
is no CPU path and no fallback: a missing library or a non-CUDA device raises.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .net import CVPIPE, PIPE, PUMP, PRV, PSV, PBV, FCV, TCV, GPV

CSMALL, CBIG, BIG, TINY, MISSING = 1e-6, 1e8, 1e10, 1e-6, -1e10
QZERO, PI = 1e-6, 3.141592654
XHEAD, TEMPCLOSED, CLOSED, OPEN, ACTIVE, XFLOW, XFCV, XPRESSURE = range(8)
MperFT, PSIperFT, KPAperPSI = 0.3048, 0.4333, 6.895
SI_FLOW_UNITS = ("LPS", "LPM", "MLD", "CMH", "CMD")
FLOW_UCF = {"CFS": 1.0, "GPM": 448.831, "MGD": 0.64632, "IMGD": 0.5382,
            "AFD": 1.9837, "LPS": 28.317, "LPM": 1699.0, "MLD": 2.4466,
            "CMH": 101.94, "CMD": 2446.6}
_LNAME = {CVPIPE: "CVPIPE", PIPE: "PIPE", PUMP: "PUMP", PRV: "PRV", PSV: "PSV",
          PBV: "PBV", FCV: "FCV", TCV: "TCV", GPV: "GPV"}


def _ptr(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class _Plan:
    """Owns one `WdsPlan*` (device tables + workspace for `max_batch`)."""

    def __init__(self, solver, max_batch):
        lib = _lib.load()
        self.lib = lib
        self.max_batch = int(max_batch)
        self.device = solver.device
        self.handle = ctypes.c_void_p()
        self.held = False                  # a pending backward keeps its terminal state here
        t = solver._tables
        self._keep = t                     # host arrays must outlive wds_plan
        net = _lib.WdsNetwork()
        net.n_nodes, net.n_links = solver.N, solver.L
        net.node_type = _ptr(t["node_type"], ctypes.c_int8)
        net.elev = _ptr(t["elev"], ctypes.c_double)
        net.link_n1 = _ptr(t["n1"], ctypes.c_int32)
        net.link_n2 = _ptr(t["n2"], ctypes.c_int32)
        net.link_kind = _ptr(t["kind"], ctypes.c_int8)
        net.link_flags = _ptr(t["flags"], ctypes.c_uint8)
        for f in ("km", "km_tcv", "q_init", "pump_h0", "pump_r", "pump_n",
                  "pump_speed", "pump_hmax", "pump_hunit", "curve_x", "curve_y", "prv_hset",
                  "tl_qsign", "tl_hmax", "tl_hmin"):
            setattr(net, f, _ptr(t[f], ctypes.c_double))
        net.status0 = _ptr(t["status0"], ctypes.c_int8)
        net.pump_type = _ptr(t["pump_type"], ctypes.c_int8)
        net.curve_ptr = _ptr(t["curve_ptr"], ctypes.c_int32)
        net.n_tank_links = int(t["tl_link"].size)
        for f in ("tl_link", "tl_tank", "tl_other"):
            setattr(net, f, _ptr(t[f], ctypes.c_int32))
        net.tl_flags = _ptr(t["tl_flags"], ctypes.c_uint8)
        net.hexp, net.qexp, net.rqtol = solver.hexp, solver.qexp, solver.rqtol
        net.htol, net.qtol = solver.htol, solver.qtol
        net.ucf_flow, net.ucf_head = solver.ucf_flow, solver.ucf_head
        net.checkfreq, net.maxcheck = solver.checkfreq, solver.maxcheck
        net.extra_iter = solver.extra_iter
        net.perm = None if solver.perm is None else _ptr(solver.perm, ctypes.c_int32)
        net.emitter_capacity = int(solver.emitter_capacity)
        net.layout = {"auto": _lib.LAYOUT_AUTO, "shared": _lib.LAYOUT_SHARED,
                      "global": _lib.LAYOUT_GLOBAL}[solver.sm100_layout]
        if solver.sm100_factor_dtype not in (torch.float64, torch.float32):
            raise ValueError("sm100_factor_dtype must be torch.float64 or torch.float32")
        net.factor_fp32 = 1 if solver.sm100_factor_dtype == torch.float32 else 0
        tun = solver.sm100_tuning or {}
        net.groups_per_cta = int(tun.get("groups_per_cta", 0))
        net.top_max = int(tun.get("top_max", 0))
        net.level_barrier_cost = float(tun.get("level_barrier_cost", 0.0))
        with torch.cuda.device(self.device):
            _lib.check(lib.wds_plan(ctypes.byref(net), self.max_batch,
                                    ctypes.byref(self.handle)), "wds_plan")

    def stats(self):
        o = np.zeros(8, dtype=np.int64)
        _lib.check(self.lib.wds_plan_stats(self.handle, _ptr(o, ctypes.c_int64)),
                   "wds_plan_stats")
        keys = ("Nj", "nnz_L", "n_levels", "n_update_pairs", "smem_bytes",
                "n_prv", "nnz_A_lower", "groups_per_cta")
        return dict(zip(keys, (int(v) for v in o)))

    def symbolic(self):
        s = self.stats()
        nj, nnz = s["Nj"], s["nnz_L"]
        perm = np.zeros(nj, np.int32)
        colptr = np.zeros(nj + 1, np.int32)
        rowidx = np.zeros(nnz, np.int32)
        parent = np.zeros(nj, np.int32)
        level = np.zeros(nj, np.int32)
        _lib.check(self.lib.wds_plan_symbolic(
            self.handle, _ptr(perm, ctypes.c_int32), _ptr(colptr, ctypes.c_int32),
            _ptr(rowidx, ctypes.c_int32), _ptr(parent, ctypes.c_int32),
            _ptr(level, ctypes.c_int32)), "wds_plan_symbolic")
        return dict(perm=perm, colptr=colptr, rowidx=rowidx, parent=parent, level=level)

    def generation(self):
        """The plan's kept-state generation (`wds_state_generation`)."""
        g = ctypes.c_int64()
        _lib.check(self.lib.wds_state_generation(self.handle, ctypes.byref(g)),
                   "wds_state_generation")
        return int(g.value)

    def free(self):
        if self.handle:
            self.lib.wds_free(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class _Hold:
    """A pending backward's claim on the plan that holds its terminal factor.

    The reference keeps the factor of each forward in its own autograd
    context (`ctx.kf`, dgga/autodiff.py:1203-1243), so two forwards before
    their backwards each differentiate their own state.  Here the factor lives
    in a plan's workspace: while a forward's backward is pending its plan is
    held, and `GGASolver.plan` gives later forwards another plan.  The claim
    ends with the backward or when the autograd graph is freed.  The plan's
    state generation, recorded at the forward, is checked before the adjoint,
    so a state that was replaced anyway (a second backward after the claim
    ended and another forward ran) raises instead of giving a wrong gradient."""

    def __init__(self, plan):
        self.plan = plan
        self.gen = plan.generation()
        self.active = True
        plan.held = True

    def check(self, who):
        if self.plan.generation() != self.gen:
            raise RuntimeError(
                "%s: the terminal state of this forward was replaced by a later forward on "
                "the same plan (backward after the graph's claim ended); run the forward "
                "again" % who)

    def release(self):
        if self.active:
            self.active = False
            self.plan.held = False

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def _not_pd_hint(solver):
    """Suffix of a not-positive-definite error in FP32-factor mode."""
    if getattr(solver, "sm100_factor_dtype", torch.float64) == torch.float32:
        return (" (sm100_factor_dtype=float32: the FP32 LDL^T lost positive "
                "definiteness on this ill-conditioned node matrix; use float64)")
    return ""


def _check_info_flags(solver, info):
    """Input errors the forward kernel reports per scenario: a NaN head at a
    reservoir/tank node (dgga/solver.py:2892-2894; the kernel solves nothing
    for that scenario) and more emitters than the plan's capacity."""
    if bool((info & _lib.INFO_BAD_HEAD).any()):
        raise ValueError("res_head_ft is nan at a reservoir/tank node")
    cap = torch.nonzero(info & _lib.INFO_EMITTER_CAP).flatten()
    if cap.numel():
        raise ValueError(
            "scenarios %s have more emitters (Ke > 0) than emitter_capacity=%d; "
            "raise solver.emitter_capacity before the first solve"
            % (cap.tolist()[:8], solver.emitter_capacity))


class GGASolver:
    """Batched GGA solver, B200 route.

    GGASolver(net, device="cuda", dtype=torch.float64, mode="dense",
              inp_path=None, dense_tank_bound_check=True,
              dense_status_machine=False)

    Same admission rules and exceptions as the reference's dense mode
    (dgga/solver.py:160-495): PIPE/TCV/PUMP (+ CVPIPE and PRV with
    `dense_status_machine=True`), Hazen-Williams or Chezy-Manning, DDA only,
    no damping, no HEADERROR/FLOWCHANGE, no junction-pressure controls, PRVs
    with a setting must join two junctions.

    `sm100_refine` is the number of iterative-refinement steps of a refined
    GGA solve (the reference's `dense_refine` / `cudss_refine` are 2).  None
    (default): 1 at accuracy >= 1e-8, where one step leaves the solve's
    rounding at about (kappa u)^2, some 1e-14 relative at config 2, nine
    orders below the convergence test; 2 at tighter accuracies, where the
    convergence test sits at the rounding floor.
    `sm100_refine_band` says which GGA iterations refine: an iteration whose
    previous relerr is below the band (or past iteration 20) refines, the
    others take one unrefined FP64 substitution, whose rounding (about 1e-11
    to 1e-9 relative) the Newton iteration corrects by itself while relerr
    is far above it.  None (default): 1e-5 with the FP64 factor at
    accuracy >= 1e-8, where that rounding is far below the convergence test
    as well; 0 (every iteration, the reference's schedule) at tighter
    accuracies and with the FP32 factor.  Polish and adjoint solves always
    refine.
    `sm100_layout` ("auto", "shared" or "global", set before the first solve)
    says where the schedule tables and per-scenario state live: shared memory
    (several scenarios per SM), or global memory for networks too large for
    it ("auto" picks shared memory when it fits).
    `sm100_factor_dtype` (torch.float64 or torch.float32, set before the first
    solve): precision of the LDL^T factor and of the substitutions; with
    float32 every linear solve is refined against the FP64 operator
    (`sm100_refine` steps), and residuals, headloss, convergence test, status
    decisions and the adjoint right-hand side stay FP64.
    """

    def __init__(self, net, device="cuda", dtype=torch.float64, mode="dense",
                 inp_path=None, dense_tank_bound_check=True,
                 dense_status_machine=False, perm=None):
        if mode not in ("epanet", "dense"):
            raise ValueError("unknown mode: %r" % (mode,))
        if mode == "epanet":
            raise NotImplementedError(
                "mode='epanet' is the reference's per-scenario EPANET replica; "
                "this package implements the batched dense route only")
        if inp_path is not None:
            raise NotImplementedError(
                "inp_path (exact EPANET property rebuild from INP text) needs "
                "the reference's INP parser; pass a Net instead")
        self.mode = mode
        self.dense_status_machine = bool(dense_status_machine)
        self.device = torch.device(device)
        self.dtype = dtype
        self.net = net
        self.sm100_refine = None
        self.sm100_refine_band = None
        self.sm100_layout = "auto"
        # schedule choices of the planner (groups_per_cta, top_max,
        # level_barrier_cost; None: its cost model), set by wdsgpu_b200.tune
        self.sm100_tuning = None
        self.sm100_factor_dtype = torch.float64
        # emitters per scenario kept in shared memory (junctions with Ke > 0)
        self.emitter_capacity = max(64, 2 * int((np.asarray(net.node_ke) > 0).sum()))
        lt = np.asarray(net.link_type, dtype=np.int64)
        nt = np.asarray(net.node_type, dtype=np.int64)
        allowed = ({CVPIPE, PIPE, TCV, PUMP, PRV, PSV, FCV} if self.dense_status_machine
                   else {PIPE, TCV, PUMP})
        bad = set(lt.tolist()) - allowed
        if bad:
            raise NotImplementedError(
                "mode=dense supports link_type in %s, got %s (%s)" % (
                    sorted(allowed), sorted(bad),
                    ", ".join(_LNAME.get(b, str(b)) for b in sorted(bad))))
        meta = net.meta
        self.headloss_form = str(meta.get("headloss", "H-W")).upper()
        if self.headloss_form not in ("H-W", "D-W", "C-M"):
            raise NotImplementedError("unknown headloss formula %s" % self.headloss_form)
        if self.headloss_form == "D-W":
            raise NotImplementedError("D-W is epanet-mode only")
        if str(meta.get("demand_model", "DDA")).upper() != "DDA":
            raise NotImplementedError("only the DDA demand model is supported")
        if float(meta.get("damp_limit", 0.0)) > 0.0:
            raise NotImplementedError("DAMPLIMIT>0 is not supported")
        if float(meta.get("headerror", 0.0)) > 0.0 or float(meta.get("flowchange", 0.0)) > 0.0:
            raise NotImplementedError("HEADERROR/FLOWCHANGE>0 convergence is not supported")
        self.N, self.L = len(nt), len(lt)
        is_junc = nt == 0
        self.junc_nodes = np.flatnonzero(is_junc)
        self.fixed_nodes = np.flatnonzero(~is_junc)
        self.Nj = int(is_junc.sum())
        self.hexp = 1.852 if self.headloss_form == "H-W" else 2.0
        self.qexp = float(meta["qexp"])
        self.rqtol = float(meta.get("rqtol", 1e-7))
        self.max_iter_default = int(meta["trials"])
        self.hacc_default = min(max(float(meta["accuracy"]), 1e-5), 1e-1)
        self.htol = float(meta.get("htol", 0.0005))
        self.qtol = float(meta.get("qtol", 0.0001))
        self.checkfreq = int(meta.get("checkfreq", 2))
        self.maxcheck = int(meta.get("maxcheck", 10))
        self.extra_iter = int(meta.get("extra_iter", -1))
        self._check_pswitch(net, nt)
        self.perm = None if perm is None else np.ascontiguousarray(perm, dtype=np.int32)
        self._build_tables(net, lt, nt)
        self.node_ke_default = torch.as_tensor(np.asarray(net.node_ke, dtype=np.float64),
                                               device=self.device)
        self.r_hw = torch.as_tensor(np.asarray(net.r_hw, dtype=np.float64), device=self.device)
        self._plans = []
        self._zeros = {}

    # ------------------------------------------------------------ set-up
    @staticmethod
    def _check_pswitch(net, nt):
        """Junction-pressure simple controls act after convergence (pswitch,
        hydsolver.c:268-355); the batched route has no counterpart, so they
        are refused at construction (dgga/solver.py:617-644)."""
        cn = np.asarray(getattr(net, "ctl_node", np.zeros(0)), dtype=np.int64)
        ct = np.asarray(getattr(net, "ctl_type", np.zeros(0)), dtype=np.int64)
        if cn.size:
            hit = (cn >= 0) & (ct < 2) & (nt[np.where(cn >= 0, cn, 0)] == 0)
            if hit.any():
                raise NotImplementedError(
                    "mode=dense: a simple control monitors a junction head "
                    "(pswitch); use the reference's mode='epanet'")

    def _build_tables(self, net, lt, nt):
        """Per-link tables derived exactly as the reference's __init__ does."""
        N, L = self.N, self.L
        meta = net.meta
        st = np.asarray(net.init_status, dtype=np.int64)
        status0 = np.array([{0: CLOSED, 1: OPEN, 2: ACTIVE}[int(s)] for s in st],
                           dtype=np.int8)
        setting = np.asarray(net.valve_setting_user, dtype=np.float64)
        diam = np.asarray(net.diam_ft, dtype=np.float64)
        km = np.asarray(net.km_int, dtype=np.float64)
        d4 = diam ** 2 * diam ** 2
        km_tcv = np.where(st == 2, np.divide(0.02517 * setting, d4,
                                             out=np.zeros_like(setting), where=d4 > 0), km)
        spg = float(meta.get("spgrav", 1.0))
        press = str(meta.get("press_units", "") or "")
        fu = str(meta["flow_units"])
        self.ucf_flow = FLOW_UCF[fu]
        if fu in SI_FLOW_UNITS:
            self.ucf_head = MperFT
            self.ucf_pressure = (MperFT * spg if (press or "METERS") != "KPA"
                                 else KPAperPSI * PSIperFT * spg)
        else:
            self.ucf_head = 1.0
            self.ucf_pressure = PSIperFT * spg
        K0 = setting.copy()
        for k in np.flatnonzero(lt >= PRV):
            if status0[k] != ACTIVE:
                K0[k] = MISSING
            elif lt[k] in (PRV, PSV, PBV):
                K0[k] = K0[k] / self.ucf_pressure
            elif lt[k] == FCV:
                K0[k] = K0[k] / self.ucf_flow
        self.init_setting = K0
        is_pump = lt == PUMP
        pl = np.asarray(net.pump_link, dtype=np.int64)
        ptype = np.full(L, -1, dtype=np.int8)
        ph0, pr, pn = np.zeros(L), np.zeros(L), np.zeros(L)
        pq0, phm = np.zeros(L), np.zeros(L)
        if pl.size:
            ptype[pl] = np.asarray(net.pump_ptype)
            ph0[pl] = np.asarray(net.pump_h0)
            pr[pl] = np.asarray(net.pump_r)
            pn[pl] = np.asarray(net.pump_n)
            pq0[pl] = np.asarray(net.pump_q0)
            phm[pl] = np.asarray(net.pump_hmax)
        pn[np.abs(pn - 1.0) < TINY] = 1.0
        sp = K0
        chp = ptype == 0
        pump_hmax = np.where(chp, BIG, sp * sp * phm)
        flags = np.zeros(L, dtype=np.uint8)
        flags |= np.where(is_pump & (sp == 0.0), _lib.F_ZERO_SPEED, 0).astype(np.uint8)
        flags |= np.where(is_pump & (sp > 0.0), _lib.F_PUMP_LIVE, 0).astype(np.uint8)
        flags |= np.where(chp, _lib.F_CHP, 0).astype(np.uint8)
        flags |= np.where(lt <= PIPE, _lib.F_IS_PIPE, 0).astype(np.uint8)
        kind = np.full(L, _lib.KIND_PIPE, dtype=np.int8)
        kind[lt == CVPIPE] = _lib.KIND_CVPIPE
        kind[lt == TCV] = _lib.KIND_TCV
        kind[is_pump] = _lib.KIND_PUMP
        prv = lt == PRV
        psv = lt == PSV
        prvs = prv & (K0 != MISSING)
        psvs = psv & (K0 != MISSING)
        pcv = prvs | psvs             # pressure control valves with a setting
        kind[(prv | psv) & ~pcv] = _lib.KIND_PRV_FIXED
        kind[prvs] = _lib.KIND_PRV
        kind[psvs] = _lib.KIND_PSV
        # FCVs with a flow setting take the valve pass and fcvstatus; a fixed
        # (MISSING setting) FCV is a fixed open/closed valve like a fixed PRV
        fcv = lt == FCV
        fcvs = fcv & (K0 != MISSING)
        kind[fcv & ~fcvs] = _lib.KIND_PRV_FIXED
        kind[fcvs] = _lib.KIND_FCV
        self.fcv_links = np.flatnonzero(fcvs)
        self.has_cv = bool((lt == CVPIPE).any())
        self.n_pcv = int(pcv.sum())
        self.pcv_links = np.flatnonzero(pcv)
        n1 = np.asarray(net.link_n1, dtype=np.int64)
        n2 = np.asarray(net.link_n2, dtype=np.int64)
        # the junction an ACTIVE valve holds (PRV n2, PSV n1) and its other end
        self.pcv_jc = np.where(psvs, n1, n2)[self.pcv_links]
        self.pcv_jo = np.where(psvs, n2, n1)[self.pcv_links]
        is_fixed = nt != 0
        if self.n_pcv:
            if self.dtype != torch.float64:
                raise NotImplementedError(
                    "mode=dense with setting PRVs/PSVs needs float64 (ACTIVE valve rows "
                    "carry a 1e8 penalty diagonal)")
            badp = self.pcv_links[is_fixed[n1[self.pcv_links]] | is_fixed[n2[self.pcv_links]]]
            if badp.size:
                raise NotImplementedError(
                    "mode=dense batched PRVs/PSVs need junctions at both ends: %s"
                    % [net.link_id[int(k)] for k in badp])
        if self.fcv_links.size:
            badf = self.fcv_links[is_fixed[n1[self.fcv_links]] | is_fixed[n2[self.fcv_links]]]
            if badf.size:
                raise NotImplementedError(
                    "mode=dense batched FCVs need junctions at both ends: %s"
                    % [net.link_id[int(k)] for k in badf])
        elev = np.asarray(net.elev_ft, dtype=np.float64)
        # valve settings: PRV head El[n2] + setting, PSV El[n1] + setting (ft),
        # FCV flow setting (cfs)
        prv_hset = np.zeros(L)
        prv_hset[prvs] = elev[n2[prvs]] + K0[prvs]
        prv_hset[psvs] = elev[n1[psvs]] + K0[psvs]
        prv_hset[fcvs] = K0[fcvs]
        # initial flows (hydraul.c initlinkflow as restated in solver.py:2163-2174)
        q = PI * diam ** 2 / 4.0
        if pl.size:
            q = np.where(is_pump, K0 * pq0, q)
        q_init = np.where(st == 0, QZERO, q)
        self._q_open = q          # initlinkflow of an open link (frozen-status warm starts)
        # custom pump curves, one range per link
        curve_ptr = np.zeros(L + 1, dtype=np.int32)
        cx, cy = [], []
        if pl.size:
            cq = np.asarray(net.pump_curve_q, dtype=np.float64)
            ch = np.asarray(net.pump_curve_h, dtype=np.float64)
            cp = np.asarray(net.pump_curve_ptr, dtype=np.int64)
            pos = {int(k): j for j, k in enumerate(pl)}
            for k in range(L):
                if k in pos and ptype[k] == 2:
                    j = pos[k]
                    xs, ys = cq[cp[j]:cp[j + 1]], ch[cp[j]:cp[j + 1]]
                    if xs.size < 2 or np.any(np.diff(xs) <= 0):
                        raise NotImplementedError(
                            "CUSTOM pump %s: curve flows must be strictly increasing "
                            "with at least two points" % net.link_id[k])
                    cx += xs.tolist()
                    cy += ys.tolist()
                curve_ptr[k + 1] = len(cx)
        else:
            curve_ptr[:] = 0
        # tank links (tankstatus, solver.py:536-568)
        tn = np.asarray(net.tank_node, dtype=np.int64)
        is_tank = np.zeros(N, dtype=bool)
        is_tank[tn] = True
        thmax, thmin = np.zeros(N), np.zeros(N)
        tovf = np.zeros(N, dtype=bool)
        if tn.size:
            thmax[tn] = np.asarray(net.tank_hmax)
            thmin[tn] = np.asarray(net.tank_hmin)
            tovf[tn] = np.asarray(net.tank_overflow) != 0
        use_n2 = (~is_fixed[n1]) & is_fixed[n2]
        cand = np.where(is_fixed[n1], n1, np.where(is_fixed[n2], n2, -1))
        sel = (cand >= 0) & is_tank[np.where(cand >= 0, cand, 0)]
        kk = np.flatnonzero(sel)
        tank = cand[kk]
        tl_flags = (np.where(tovf[tank], _lib.TL_OVERFLOW, 0)
                    | np.where(is_pump[kk], _lib.TL_IS_PUMP, 0)
                    | np.where(is_pump[kk] & (n2[kk] == tank), _lib.TL_PUMP_IN, 0)
                    | np.where(is_pump[kk] & (n1[kk] == tank), _lib.TL_PUMP_OUT, 0)
                    ).astype(np.uint8)
        c64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        c32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        self._tables = dict(
            node_type=np.ascontiguousarray(nt, dtype=np.int8), elev=c64(elev),
            n1=c32(n1), n2=c32(n2), kind=kind, flags=flags, km=c64(km),
            km_tcv=c64(km_tcv), q_init=c64(q_init), status0=status0,
            pump_type=ptype, pump_h0=c64(ph0), pump_r=c64(pr), pump_n=c64(pn),
            pump_speed=c64(sp), pump_hmax=c64(pump_hmax),
            pump_hunit=c64(np.where(chp, BIG, phm)), curve_ptr=curve_ptr,
            curve_x=c64(cx if cx else [0.0]), curve_y=c64(cy if cy else [0.0]),
            prv_hset=c64(prv_hset), tl_link=c32(kk), tl_tank=c32(tank),
            tl_other=c32(np.where(use_n2[kk], n1[kk], n2[kk])),
            tl_qsign=c64(np.where(use_n2[kk], -1.0, 1.0)), tl_hmax=c64(thmax[tank]),
            tl_hmin=c64(thmin[tank]), tl_flags=tl_flags)
        self._tank = dict(k=kk, tank=tank, other=np.where(use_n2[kk], n1[kk], n2[kk]),
                          qsign=np.where(use_n2[kk], -1.0, 1.0), hmax=thmax[tank],
                          hmin=thmin[tank], ovf=tovf[tank], is_pump=is_pump[kk],
                          pin=is_pump[kk] & (n2[kk] == tank),
                          pout=is_pump[kk] & (n1[kk] == tank), live=st[kk] != 0)
        self._pump = dict(links=pl, n1=n1[pl] if pl.size else pl, n2=n2[pl] if pl.size else pl,
                          hmax=pump_hmax[pl] if pl.size else np.zeros(0),
                          live=((~(st == 0)) & ~(sp == 0.0))[pl] if pl.size else np.zeros(0, bool))
        self._n1, self._n2 = n1, n2
        self._lt = lt

    # Optional launch timing: when `launch_events` is a list, every C-ABI
    # launch appends (name, start_event, end_event) recorded on the launching
    # stream around the call.
    launch_events = None

    def _event_pair(self, stream, name):
        if self.launch_events is None:
            return None
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        self.launch_events.append((name, e0, e1))
        return e0, e1

    def plan(self, batch):
        """Plan (symbolic analysis + device tables + workspace) able to run
        `batch` scenarios: the smallest kept plan of enough capacity whose
        terminal state no pending backward holds, else a new one (capacity a
        power of two)."""
        if self.device.type != "cuda":
            raise NotImplementedError(
                "linear_solver='sm100' needs a CUDA device (got %s)" % self.device)
        free = [p for p in self._plans if p.max_batch >= batch and not p.held]
        if free:
            return min(free, key=lambda p: p.max_batch)
        cap = 1
        while cap < batch:
            cap *= 2
        p = _Plan(self, cap)
        self._plans.append(p)
        return p

    def plan_stats(self, batch=1):
        return self.plan(batch).stats()

    def symbolic(self):
        return self.plan(1).symbolic()

    # ------------------------------------------------------------ solve
    def _zero_rows(self, B, n):
        """A cached [B, n] float64 block of zeros on the solver's device, for
        read-only inputs of the C ABI (an output adjoint that autograd left
        as None); never written."""
        key = (int(B), int(n))
        z = self._zeros.get(key)
        if z is None:
            z = torch.zeros(key, dtype=torch.float64, device=self.device)
            self._zeros[key] = z
        return z

    def _cvt(self, x):
        if isinstance(x, torch.Tensor):
            return x.to(dtype=torch.float64, device=self.device)
        return torch.as_tensor(np.asarray(x), dtype=torch.float64, device=self.device)

    def _inputs(self, demand, res_head, ke, r):
        d = self._cvt(demand)
        rh = self._cvt(res_head)
        single = d.dim() == 1
        d = d.unsqueeze(0) if single else d
        rh = rh.unsqueeze(0) if rh.dim() == 1 else rh
        B = d.shape[0]
        if rh.shape[0] == 1 and B > 1:
            rh = rh.expand(B, -1)
        if d.shape[1] != self.N or rh.shape[1] != self.N:
            raise ValueError("demand/res_head must have N=%d columns" % self.N)
        ke = self.node_ke_default if ke is None else self._cvt(ke)
        ke = ke.unsqueeze(0) if ke.dim() == 1 else ke
        r = self.r_hw if r is None else self._cvt(r)
        r = r.unsqueeze(0) if r.dim() == 1 else r
        if ke.shape[0] not in (1, B) or r.shape[0] not in (1, B):
            raise ValueError("ke / r_hw must be [N] / [L] or batched like demand")
        d = d.contiguous()
        rh = rh.contiguous()
        ke = ke.contiguous()
        r = r.contiguous()
        # a NaN reservoir/tank head is reported by the forward kernel (info
        # WDS_INFO_BAD_HEAD, raised by _check_info_flags), so that the inputs
        # cost no host synchronisation before the launch
        return d, rh, ke, r, B, single

    def _guards(self, status_machine, assemble, linear_solver, link_status,
                link_setting, record_schedule):
        if assemble not in ("dense", "csr"):
            raise ValueError("assemble must be 'dense'/'csr', got %r" % (assemble,))
        if linear_solver not in ("dense", "cudss", "sm100"):
            raise ValueError("linear_solver must be 'dense'/'cudss'/'sm100', got %r"
                             % (linear_solver,))
        if linear_solver != "sm100":
            raise NotImplementedError(
                "this package provides linear_solver='sm100' only; the 'dense' "
                "and 'cudss' routes are the reference's own")
        if assemble != "csr":
            raise ValueError("linear_solver='sm100' needs assemble='csr', got %r" % (assemble,))
        if self.dtype != torch.float64:
            raise NotImplementedError("linear_solver='sm100' keeps the state in float64")
        if not self.dense_status_machine:
            if link_status is not None or link_setting is not None or status_machine:
                raise NotImplementedError(
                    "link_status/link_setting/status_machine need "
                    "dense_status_machine=True at construction")
        else:
            if link_status is not None or link_setting is not None:
                raise NotImplementedError(
                    "the batched status machine starts from the initial "
                    "configuration; link_status/link_setting are epanet-mode only")
            if self.has_cv and not status_machine:
                raise NotImplementedError(
                    "this network has CVPIPEs: solve(..., status_machine=True) is required")
            if (self.n_pcv or self.fcv_links.size) and not status_machine:
                raise NotImplementedError(
                    "this network has PRVs/PSVs/FCVs with a setting: solve(..., "
                    "status_machine=True) is required")
        if record_schedule and not status_machine:
            raise ValueError(
                "record_schedule=True covers the batched status machine only "
                "(status_machine=True), as in the reference")

    def refine_steps(self, accuracy=None):
        """Refinement steps of a refined GGA solve (`sm100_refine`; None: 1 at
        accuracy >= 1e-8, else 2)."""
        if self.sm100_refine is not None:
            return int(self.sm100_refine)
        return 1 if accuracy is not None and float(accuracy) >= 1e-8 else 2

    def refine_band(self, accuracy):
        """Refinement band of the GGA iterations (see `sm100_refine_band`)."""
        if self.sm100_refine_band is not None:
            return float(self.sm100_refine_band)
        if self.sm100_factor_dtype == torch.float32 or float(accuracy) < 1e-8:
            return 0.0
        return 1e-5

    def pump_rows(self, B, speed=None, pump_h0=None, pump_r=None):
        """Pump parameters of a call as FP64 device rows: (speed, h0, r), each
        None or [1, L] / [B, L] with one common row count (an [L] row next to
        [B, L] rows is expanded).  Values off pump links are not read."""
        vals = [speed, pump_h0, pump_r]
        if all(v is None for v in vals):
            return None
        dev, L = self.device, self.L
        out = []
        for name, v in zip(("speed", "pump_h0", "pump_r"), vals):
            if v is None:
                out.append(None)
                continue
            t = v.detach() if isinstance(v, torch.Tensor) else torch.as_tensor(np.asarray(v))
            t = t.to(dtype=torch.float64, device=dev)
            if t.dim() == 1:
                t = t.unsqueeze(0)
            if t.dim() != 2 or t.shape[1] != L or t.shape[0] not in (1, B):
                raise ValueError("%s must be [L] or [B, L] (L=%d, B=%d), got %s"
                                 % (name, L, B, tuple(t.shape)))
            if name == "speed":
                # the reference's speed is the whole link-setting vector
                # (LinkSetting, dgga/autodiff.py:99-120); off pump links it
                # would set valve settings, which this route does not take
                off = self._lt != PUMP
                host = t.cpu().numpy()
                bad = np.flatnonzero((host[:, off] != self.init_setting[off]).any(0))
                if bad.size:
                    raise NotImplementedError(
                        "speed differs from the network's link settings off pump links "
                        "(links %s): valve settings are not parameters of this route"
                        % np.flatnonzero(off)[bad][:8].tolist())
            out.append(t)
        rows = max(t.shape[0] for t in out if t is not None)
        return tuple(None if t is None else t.expand(rows, L).contiguous() for t in out)

    def run(self, d, rh, ke, r, B, max_iter, hacc, status_machine, polish_steps,
            refine=None, plan=None, q0=None, e0=None, pumps=None, refine_band=None,
            record=None, schedule=False, S0=None):
        """One wds_forward call on device tensors; returns the raw outputs.
        q0 [B,L] / e0 [B,N] (contiguous FP64 on the device, or None) are the
        warm start of GGASolver.solve (dgga/solver.py:2876-2887); pumps is
        the (speed, h0, r) of `pump_rows` (the call's pump parameters, or
        None for the network's).  The result holds `diag_ratio` [B] on networks
        with status-machine PRVs/PSVs, and with schedule=True the raw schedule
        record (`sched_flags`, `sched_chg`) for `_schedule`."""
        p = plan or self.plan(B)
        dev = self.device
        head = torch.empty(B, self.N, dtype=torch.float64, device=dev)
        flow = torch.empty(B, self.L, dtype=torch.float64, device=dev)
        emit = torch.empty(B, self.N, dtype=torch.float64, device=dev)
        status = torch.empty(B, self.L, dtype=torch.int8, device=dev)
        iters = torch.empty(B, dtype=torch.int32, device=dev)
        relerr = torch.empty(B, dtype=torch.float64, device=dev)
        info = torch.empty(B, dtype=torch.int32, device=dev)
        o = _lib.WdsForwardOpts()
        o.accuracy = float(hacc)
        o.max_iter = int(max_iter)
        o.status_machine = 1 if status_machine else 0
        o.refine = int(self.refine_steps(hacc) if refine is None else refine)
        o.refine_band = float(self.refine_band(hacc) if refine_band is None else refine_band)
        if record is not None:   # unrolled mode: max_iter iterations, recorded
            o.unroll_record = record.data_ptr()
        diag = None
        if self.n_pcv:
            diag = torch.zeros(B, dtype=torch.float64, device=dev)
            o.diag_ratio = diag.data_ptr()
        sflags = schg = None
        if schedule:
            T = int(max_iter) + max(int(self.extra_iter), 0)
            sflags = torch.zeros(B, T, dtype=torch.uint8, device=dev)
            schg = torch.zeros(B, T, (self.L + 31) // 32, dtype=torch.int32, device=dev)
            o.sched_flags, o.sched_chg = sflags.data_ptr(), schg.data_ptr()
        o.polish_steps = int(polish_steps)
        o.ke_stride = 0 if ke.shape[0] == 1 else self.N
        o.r_stride = 0 if r.shape[0] == 1 else self.L
        if S0 is not None:       # status warm start (extended-period steps)
            if S0.dtype != torch.int8 or not S0.is_contiguous() or tuple(S0.shape) != (B, self.L):
                raise ValueError("S0 must be a contiguous int8 [%d, %d] tensor" % (B, self.L))
            o.status0 = S0.data_ptr()
        for name, t, cols in (("q0", q0, self.L), ("e0", e0, self.N)):
            if t is not None:
                same_dev = t.device.type == dev.type and (dev.index is None
                                                          or t.device.index == dev.index)
                if (t.dtype != torch.float64 or not same_dev or not t.is_contiguous()
                        or tuple(t.shape) != (B, cols)):
                    raise ValueError("%s must be a contiguous float64 [%d, %d] tensor on %s"
                                     % (name, B, cols, dev))
                setattr(o, name, t.data_ptr())
        if pumps is not None:
            rows = next(t.shape[0] for t in pumps if t is not None)
            o.pump_stride = 0 if rows == 1 else self.L
            for name, t in zip(("pump_speed", "pump_h0", "pump_r"), pumps):
                if t is not None:
                    setattr(o, name, t.data_ptr())
        cur = torch.cuda.current_stream(dev)
        stream = cur.cuda_stream
        ev = self._event_pair(cur, "forward")
        _lib.check(p.lib.wds_forward(
            p.handle, B, ctypes.byref(o), d.data_ptr(), rh.data_ptr(), ke.data_ptr(),
            r.data_ptr(), head.data_ptr(), flow.data_ptr(), emit.data_ptr(),
            status.data_ptr(), iters.data_ptr(), relerr.data_ptr(), info.data_ptr(),
            ctypes.c_void_p(stream)), "wds_forward")
        if ev is not None:
            ev[1].record(cur)
        return dict(head=head, flow=flow, emit=emit, status=status, iters=iters,
                    relerr=relerr, info=info, plan=p, pumps=pumps, diag_ratio=diag,
                    sched_flags=sflags, sched_chg=schg)

    def _schedule(self, flags, chg):
        """The schedule list of the reference (dgga/solver.py:3136-3160): per
        iteration that any scenario ran, on networks with status-machine
        valves, dict(it, kind="valve", act[B], chg[B,L]) for the valve status
        pass, then, when any scenario ran the link-status check,
        dict(it, conv[B], per[B], chg[B,L])."""
        fl = flags.cpu().numpy()
        bits = chg.cpu().numpy().view(np.uint8)
        valve = np.zeros(self.L, dtype=bool)
        valve[self.pcv_links] = True
        out = []
        for t in np.flatnonzero((fl & 4).any(0)):
            act = (fl[:, t] & 4) != 0
            conv = (fl[:, t] & 1) != 0
            per = (fl[:, t] & 2) != 0
            c = np.unpackbits(bits[:, t, :], axis=1, bitorder="little")[:, :self.L].astype(bool)
            if self.n_pcv:
                out.append(dict(it=int(t) + 1, kind="valve", act=act,
                                chg=c & valve[None, :] & act[:, None]))
            if (conv | per).any():
                out.append(dict(it=int(t) + 1, conv=conv, per=per,
                                chg=c & ~valve[None, :] & (conv | per)[:, None]))
        return out

    def solve(self, demand_cfs, res_head_ft, ke_int=None, q0=None, e0=None,
              max_iter=None, accuracy=None, link_status=None, link_setting=None,
              status_machine=False, assemble="csr", linear_solver="sm100",
              record_schedule=False, r_hw=None):
        """Batched steady solve (dgga/solver.py:2703-3212 contract).

        Returns dict(head_ft[B,N], flow_cfs[B,L], emitter_cfs[B,N],
        iters int64[B], relerr[B], converged bool[B][, status int8[B,L]]);
        1-D demand gives unbatched outputs.  Unconverged scenarios report
        maxtrials+1 and converged=False; a non-positive pivot raises
        RuntimeError naming the scenarios."""
        self._guards(status_machine, assemble, linear_solver, link_status,
                     link_setting, record_schedule)
        d, rh, ke, r, B, single = self._inputs(demand_cfs, res_head_ft, ke_int, r_hw)
        q0 = self._warm(q0, B, self.L)
        e0 = self._warm(e0, B, self.N)
        max_iter = self.max_iter_default if max_iter is None else int(max_iter)
        hacc = self.hacc_default if accuracy is None else float(accuracy)
        sm = bool(status_machine)
        o = self.run(d, rh, ke, r, B, max_iter, hacc, sm, -1, q0=q0, e0=e0,
                     schedule=bool(record_schedule))
        info = o["info"]
        _check_info_flags(self, info)
        bad = torch.nonzero(info & _lib.INFO_NOT_PD).flatten()
        if bad.numel():
            raise RuntimeError(
                "batched LDL^T failed: the node matrix of scenarios %s is not "
                "positive definite%s" % (bad.tolist(), _not_pd_hint(self)))
        out = dict(head_ft=o["head"], flow_cfs=o["flow"], emitter_cfs=o["emit"],
                   iters=o["iters"].to(torch.int64), relerr=o["relerr"],
                   converged=(info == 0))
        if sm:
            out["status"] = o["status"]
        else:
            self._check_pump_shutoff(o["head"], o["flow"])
            self._check_tank_status(o["head"], o["flow"])
        if o["diag_ratio"] is not None:
            out["diag_ratio"] = o["diag_ratio"]
        if single:
            out = {k: v[0] for k, v in out.items()}
        if record_schedule:   # a list, not batched
            out["schedule"] = self._schedule(o["sched_flags"], o["sched_chg"])
        return out

    def _warm(self, x, B, cols):
        """A 1-D or [B, cols] warm start as a contiguous [B, cols] FP64 device
        tensor (the reference expands a 1-D q0/e0 over the batch,
        solver.py:2878-2887)."""
        if x is None:
            return None
        t = torch.as_tensor(x, dtype=torch.float64, device=self.device)
        if t.dim() == 1:
            t = t.unsqueeze(0).expand(B, -1)
        if tuple(t.shape) != (B, cols):
            raise ValueError("warm start must have shape [%d] or [%d, %d]" % (cols, B, cols))
        return t.contiguous()

    # ------------------------------------------------------------ post checks
    def _check_pump_shutoff(self, H, q):
        """Without the status machine a pump that EPANET would shut (XHEAD)
        is an error, never silently kept open (dgga/solver.py:2328-2366)."""
        pp = self._pump
        if not pp["links"].size or not pp["live"].any():
            return
        dev = H.device
        n1 = torch.as_tensor(pp["n1"], device=dev)
        n2 = torch.as_tensor(pp["n2"], device=dev)
        gain = H.index_select(1, n2) - H.index_select(1, n1)
        hmax = torch.as_tensor(pp["hmax"], dtype=H.dtype, device=dev)
        live = torch.as_tensor(pp["live"], device=dev)
        hit = (gain > hmax + self.htol) & live
        if bool(hit.any()):
            b, j = [int(x) for x in torch.nonzero(hit)[0]]
            raise NotImplementedError(
                "mode=dense: scenario b=%d pump %s exceeds its shut-off head; "
                "EPANET would close it (XHEAD). Use status_machine=True."
                % (b, self.net.link_id[int(pp["links"][j])]))

    def _check_tank_status(self, H, q):
        """Without the status machine a full/empty tank that would close its
        link is an error (dgga/solver.py:570-615)."""
        t = self._tank
        if not t["k"].size:
            return
        dev = H.device
        T = lambda a, dt=None: torch.as_tensor(a, device=dev, dtype=dt)
        live = T(t["live"])
        ht = H.index_select(1, T(t["tank"]))
        dh = ht - H.index_select(1, T(t["other"]))
        qk = q.index_select(1, T(t["k"])) * T(t["qsign"], H.dtype)
        big = dh.abs() > self.htol
        cbig = (dh < -self.htol) | (qk < -self.qtol)
        cl_open = torch.where(big, cbig, qk < -self.qtol)
        cl_closed = torch.where(big, cbig, torch.ones_like(cbig))
        full = (ht >= T(t["hmax"], H.dtype) - self.htol) & ~T(t["ovf"])
        empty = ht <= T(t["hmin"], H.dtype) + self.htol
        isp = T(t["is_pump"])
        cut_f = torch.where(isp, T(t["pin"]), cl_open)
        cut_e = torch.where(isp, T(t["pout"]), ~cl_closed)
        hit = live & ((full & cut_f) | (empty & cut_e))
        if bool(hit.any()):
            b, j = [int(x) for x in torch.nonzero(hit)[0]]
            raise NotImplementedError(
                "mode=dense: scenario b=%d tank %s is full/empty and would close "
                "link %s (tankstatus). Use status_machine=True."
                % (b, self.net.node_id[int(t["tank"][j])],
                   self.net.link_id[int(t["k"][j])]))
