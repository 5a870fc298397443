"""Implicit-function adjoint on the B200 route.

`implicit_solve(..., adjoint="gpu")` mirrors the reference entry point
(dgga/autodiff.py:1315-1351) and `ImplicitGGASolveSM100` mirrors
`ImplicitGGASolveGPU` (dgga/autodiff.py:1157-1312):

* forward: one `wds_forward` launch runs the GGA loop with the batched status
  machine, `polish_steps` reduced Newton steps (Woodbury row replacement for
  ACTIVE PRVs) and a terminal factorisation kept in the plan's workspace;
* backward: one `wds_adjoint` launch solves the reduced node adjoint on that
  terminal factor (zero new factorisations) and contracts it into
  dL/d(demand, reservoir head, emitter Ke, pipe resistance).  1-D parameters
  receive the batch-summed gradient (dgga/autodiff.py:1306-1308).

Pump parameters (speed, pump_h0, pump_r) are differentiable here too: the
forward keeps d hloss / d theta of every pump at the terminal state and
`wds_adjoint_pumps` contracts it with the link adjoint, the formulas of the
reference's CPU adjoint (dgga/autodiff.py:122-218, 736-741).

Constant-HP pumps on their CBIG / RQtol clamp branch, which the reference's
GPU route refuses (its assembled +hgrad is not the exact -hgrad of the CPU
adjoint, dgga/autodiff.py:186-193), are differentiated exactly: a Woodbury
correction on the kept factor (`_clamp_rhs`), only when such a pump exists.

Refusals follow the reference: unconverged scenarios, second derivatives,
a frozen `status`, PRVs that share a downstream junction or cascade.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .solver import CBIG, GGASolver, _Hold, _not_pd_hint

__all__ = ["implicit_solve", "ImplicitGGASolveSM100", "solve_unrolled", "UnrolledSM100",
           "unrolled_grad_health", "hw_resistance", "dr_dC"]


def _adjoint_guards(s: GGASolver, flow, S, pumps=None, allow_clamp=False):
    """Refusals of the reduced adjoint (dgga/autodiff.py:1157-1170); pumps is
    the call's (speed, h0, r) rows of GGASolver.pump_rows, or None.

    Open constant-HP pumps on their CBIG / RQtol clamp branch
    (hydcoeffs.c:748-757) are refused unless allow_clamp; then the clamped
    entries are returned as (scenario, link, assembled P) tensors (None when
    there are none) for `_clamp_rhs`."""
    if s.n_pcv and not getattr(s, "_pcv_guards_ok", False):
        # the junction each PRV (n2) or PSV (n1) holds, and its other end
        # (static per network: checked once)
        jc, jo = s.pcv_jc, s.pcv_jo
        if np.unique(jc).size < jc.size:
            raise NotImplementedError(
                "adjoint='gpu': several PRVs/PSVs hold one junction")
        if np.intersect1d(jc, jo).size:
            raise NotImplementedError(
                "adjoint='gpu': cascaded PRVs/PSVs (a held junction is another "
                "valve's other end)")
        s._pcv_guards_ok = True
    chp = s._tables["pump_type"] == 0
    if not chp.any():
        return None
    t = s._tables
    ks = np.flatnonzero(chp)
    dev = flow.device
    kt = torch.as_tensor(ks, device=dev)
    q = flow.index_select(1, kt)
    sgn = torch.where(q < 0, -1.0, 1.0)
    qa = (q * sgn).clamp_min(1e-30)
    sp_row = (pumps[0].index_select(1, kt) if pumps is not None and pumps[0] is not None
              else torch.as_tensor(t["pump_speed"][ks], device=dev))
    r_row = (pumps[2].index_select(1, kt) if pumps is not None and pumps[2] is not None
             else torch.as_tensor(t["pump_r"][ks], device=dev))
    sp = sp_row.clamp_min(1e-12)
    re = r_row * sp ** (2.0 - torch.as_tensor(t["pump_n"][ks], device=dev))
    raw = -re / qa / qa
    closed = (S.index_select(1, kt) <= 2) | (sp_row == 0.0)
    big = ~closed & (raw > CBIG)
    bad = big | (~closed & (raw < s.rqtol))
    if not bool(bad.any()):
        return None
    if not allow_clamp:
        raise NotImplementedError(
            "adjoint='gpu': a constant-HP pump sits on its CBIG/RQtol clamp "
            "branch at the converged state")
    b_idx, j_idx = torch.nonzero(bad, as_tuple=True)
    pf = torch.where(big[b_idx, j_idx], 1.0 / CBIG, 1.0 / s.rqtol).to(torch.float64)
    return b_idx, kt[j_idx], pf


def _clamp_rhs(s: GGASolver, plan, B, clamp, gH, gQ, gE, stream):
    """Adjoint right-hand side for clamped constant-HP pumps.

    On the clamp branch hloss = -hgrad q, so the exact Jacobian of the CPU
    adjoint has -hgrad where the kept factor assembled +hgrad
    (dgga/autodiff.py:186-193): the true reduced operator is the kept one
    plus sum_c dP_c a_c a_c^T (a_c the link's junction incidence,
    dP_c = -2 P_c).  By Woodbury, lambda_true = M^{-1}(r - U z) with
    z = (diag(1/dP) + V^T X)^{-1} V^T lambda, X = M^{-1} a_c (one kept-factor
    solve per clamped pump, `wds_adjoint_rhs`) and lambda = M^{-1} r (one
    `wds_adjoint`).  Since r = B^T P gQ - em gE / hge - gH, the returned gH' =
    gH + U z makes the next adjoint launch produce every gradient from
    lambda_true.  Also returns (b, k, dP) for `_clamp_grh`."""
    b_idx, k_idx, pf = clamp
    dev = gH.device
    N, L = s.N, s.L
    dP = -2.0 * pf
    # lambda of the kept operator: gd holds it at the junctions (0 at fixed nodes)
    lam = torch.empty(B, N, dtype=torch.float64, device=dev)
    t1, t2, t3 = torch.empty_like(lam), torch.empty_like(lam), torch.empty(B, L, dtype=torch.float64,
                                                                           device=dev)
    _lib.check(plan.lib.wds_adjoint(
        plan.handle, B, gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), lam.data_ptr(),
        t1.data_ptr(), t2.data_ptr(), t3.data_ptr(), ctypes.c_void_p(stream)), "wds_adjoint")
    cnt = torch.bincount(b_idx, minlength=B)
    cmax = int(cnt.max())
    first = torch.cumsum(cnt, 0) - cnt
    j_idx = torch.arange(b_idx.numel(), device=dev) - first[b_idx]
    n1 = torch.as_tensor(s._n1, device=dev)[k_idx]
    n2 = torch.as_tensor(s._n2, device=dev)[k_idx]
    junc = torch.as_tensor(s._tables["node_type"] == 0, device=dev)
    m1 = junc[n1].to(torch.float64)
    m2 = junc[n2].to(torch.float64)
    # columns x_c = M^{-1} a_c, rows b * cmax + j of wds_adjoint_rhs (gH = -a_c)
    R = B * cmax
    X = torch.empty(R, N, dtype=torch.float64, device=dev)
    v = b_idx * cmax + j_idx
    cap = plan.max_batch
    for v0 in range(0, R, cap):
        nb = min(cap, R - v0)
        gHx = torch.zeros(nb, N, dtype=torch.float64, device=dev)
        sel = (v >= v0) & (v < v0 + nb)
        vv = v[sel] - v0
        gHx.index_put_((vv, n1[sel]), -m1[sel], accumulate=True)
        gHx.index_put_((vv, n2[sel]), m2[sel], accumulate=True)
        z0 = torch.zeros(nb, L, dtype=torch.float64, device=dev)
        zN = torch.zeros(nb, N, dtype=torch.float64, device=dev)
        o1, o2 = torch.empty_like(zN), torch.empty_like(zN)
        o3 = torch.empty_like(z0)
        _lib.check(plan.lib.wds_adjoint_rhs(
            plan.handle, nb, cmax, v0, gHx.data_ptr(), z0.data_ptr(), zN.data_ptr(),
            X[v0:v0 + nb].data_ptr(), o1.data_ptr(), o2.data_ptr(), o3.data_ptr(),
            ctypes.c_void_p(stream)), "wds_adjoint_rhs")
    Xr = X.view(B, cmax, N)
    # G[b, i, j] = a_i^T x_j; padded entries get a unit diagonal and a zero rhs
    G = torch.zeros(B, cmax, cmax, dtype=torch.float64, device=dev)
    G[b_idx, j_idx, :] = Xr[b_idx, :, n1] * m1[:, None] - Xr[b_idx, :, n2] * m2[:, None]
    dg = torch.ones(B, cmax, dtype=torch.float64, device=dev)
    dg[b_idx, j_idx] = 1.0 / dP
    rhs = torch.zeros(B, cmax, dtype=torch.float64, device=dev)
    rhs[b_idx, j_idx] = lam[b_idx, n1] * m1 - lam[b_idx, n2] * m2
    z = torch.linalg.solve(G + torch.diag_embed(dg), rhs.unsqueeze(-1)).squeeze(-1)
    zc = z[b_idx, j_idx]
    gH2 = gH.clone()
    gH2.index_put_((b_idx, n1), zc * m1, accumulate=True)
    gH2.index_put_((b_idx, n2), -zc * m2, accumulate=True)
    return gH2, (b_idx, k_idx, dP, n1, n2, m1, m2)


def _clamp_grh(fix, gQ, gd, grh):
    """The clamped pump's own link adjoint lambda_l = P (gQ - (l2 - l1)) enters
    the reservoir-head gradient at a fixed endpoint; the adjoint launch formed
    it with the assembled P, so add dP (gQ - (l2 - l1)) there (+ at n1, - at
    n2, dgga/autodiff.py:726-732)."""
    b_idx, k_idx, dP, n1, n2, m1, m2 = fix
    l1 = gd[b_idx, n1] * m1
    l2 = gd[b_idx, n2] * m2
    corr = dP * (gQ[b_idx, k_idx] - (l2 - l1))
    grh.index_put_((b_idx, n1), corr * (1.0 - m1), accumulate=True)
    grh.index_put_((b_idx, n2), -corr * (1.0 - m2), accumulate=True)


class ImplicitGGASolveSM100(torch.autograd.Function):
    """(demand, res_head, ke, r_hw, solver, accuracy, max_iter, status_machine,
    polish_steps[, speed, pump_h0, pump_r]) -> (head[B,N], flow[B,L],
    emitter[B,N]).  speed / pump_h0 / pump_r ([L] shared by the batch, or
    [B,L]) are differentiable like the CPU adjoint's pump theta
    (dgga/autodiff.py:609-756); an [L] parameter receives the batch sum."""

    @staticmethod
    def forward(ctx, demand, res_head, ke, r_hw, solver, accuracy=1e-12,
                max_iter=200, status_machine=None, polish_steps=3, speed=None,
                pump_h0=None, pump_r=None):
        s = solver
        dims = (demand.dim(), res_head.dim(), ke.dim(), r_hw.dim())
        devs = (demand.device, res_head.device, ke.device, r_hw.device)
        sm = s.dense_status_machine if status_machine is None else bool(status_machine)
        s._guards(sm, "csr", "sm100", None, None, False)
        d, rh, ke_t, r_t, B, _ = s._inputs(demand.detach(), res_head.detach(),
                                           ke.detach(), r_hw.detach())
        if ke_t.shape[0] == 1 and B > 1:
            ke_t = ke_t.contiguous()
        th_in = (speed, pump_h0, pump_r)
        pumps = s.pump_rows(B, *th_in)
        o = s.run(d, rh, ke_t, r_t, B, int(max_iter), float(accuracy), sm, int(polish_steps),
                  pumps=pumps)
        info = o["info"]
        if bool((info != 0).any()):   # one host sync when every scenario converged
            from .solver import _check_info_flags
            _check_info_flags(s, info)
            bad = torch.nonzero(info != 0).flatten().tolist()
            np_ = torch.nonzero(info & _lib.INFO_NOT_PD).flatten().tolist()
            if np_:
                raise RuntimeError(
                    "adjoint='gpu': the node matrix of scenarios %s is not positive "
                    "definite%s" % (np_[:8], _not_pd_hint(s)))
            raise RuntimeError(
                "adjoint='gpu': scenarios %s did not converge (relerr=%s > accuracy=%g)"
                % (bad[:8], [float(o["relerr"][b]) for b in bad[:4]], float(accuracy)))
        ctx.clamp = _adjoint_guards(s, o["flow"], o["status"], pumps, allow_clamp=True)
        ctx.solver = s
        ctx.pumps = pumps      # keeps the rows alive with the kept state
        ctx.th = tuple(None if x is None else (x.dim(), x.device) for x in th_in)
        ctx.plan = o["plan"]
        ctx.hold = _Hold(o["plan"])   # later forwards take another plan until the backward
        ctx.B = B
        ctx.dims = dims
        ctx.devs = devs
        ctx.L = s.L
        head, flow, emit = o["head"], o["flow"], o["emit"]
        if all(x == 1 for x in dims[:3]):
            head, flow, emit = head[0], flow[0], emit[0]
        return head, flow, emit

    @staticmethod
    def backward(ctx, gH, gQ, gE):
        if torch.is_grad_enabled():
            raise NotImplementedError(
                "adjoint='gpu' is first order only (create_graph / second "
                "derivatives are not supported)")
        s = ctx.solver
        B, dev = ctx.B, s.device
        N, L = s.N, s.L

        def _g(g, n):
            if g is None:   # a read-only input of the adjoint: one cached zero block
                return s._zero_rows(B, n)
            g = g.detach().to(dtype=torch.float64, device=dev)
            g = g.unsqueeze(0).expand(B, -1) if g.dim() == 1 else g
            return g.contiguous()

        gH, gQ, gE = _g(gH, N), _g(gQ, L), _g(gE, N)
        gd = torch.empty(B, N, dtype=torch.float64, device=dev)
        grh = torch.empty_like(gd)
        gke = torch.empty_like(gd)
        gr = torch.empty(B, L, dtype=torch.float64, device=dev)
        p = ctx.plan
        ctx.hold.check("implicit_solve backward")
        cur = torch.cuda.current_stream(dev)
        ev = s._event_pair(cur, "adjoint")
        fix = None
        if ctx.clamp is not None:
            gH, fix = _clamp_rhs(s, p, B, ctx.clamp, gH, gQ, gE, cur.cuda_stream)
        want_th = any(x is not None for x in ctx.th) and any(ctx.needs_input_grad[9:12])
        if want_th:
            gth = torch.empty(3, B, L, dtype=torch.float64, device=dev)
            _lib.check(p.lib.wds_adjoint_pumps(
                p.handle, B, gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), gd.data_ptr(),
                grh.data_ptr(), gke.data_ptr(), gr.data_ptr(), gth[0].data_ptr(),
                gth[1].data_ptr(), gth[2].data_ptr(), ctypes.c_void_p(cur.cuda_stream)),
                "wds_adjoint_pumps")
        else:
            _lib.check(p.lib.wds_adjoint(
                p.handle, B, gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), gd.data_ptr(),
                grh.data_ptr(), gke.data_ptr(), gr.data_ptr(), ctypes.c_void_p(cur.cuda_stream)),
                "wds_adjoint")
        ctx.hold.release()   # stream order keeps the adjoint ahead of a later forward
        if fix is not None:
            _clamp_grh(fix, gQ, gd, grh)
        if ev is not None:
            ev[1].record(cur)
        dm, dv = ctx.dims, ctx.devs

        def _fit(g, dim, d_):
            g = g.to(device=d_)
            return g.sum(0) if dim == 1 else g

        g_th = [None, None, None]
        if want_th:
            for i, meta in enumerate(ctx.th):
                if meta is not None and ctx.needs_input_grad[9 + i]:
                    g_th[i] = _fit(gth[i], meta[0], meta[1])
        return (_fit(gd, dm[0], dv[0]), _fit(grh, dm[1], dv[1]), _fit(gke, dm[2], dv[2]),
                _fit(gr, dm[3] + 1, dv[3]), None, None, None, None, None, *g_th)


def implicit_solve(solver, demand, res_head, ke=None, r_hw=None, accuracy=1e-12,
                   max_iter=200, polish_steps=3, speed=None, pump_h0=None, pump_r=None,
                   status=None, adjoint="gpu", status_machine=None, assemble="csr",
                   linear_solver="sm100"):
    """Forward + implicit adjoint (dgga/autodiff.py:1315-1351 contract).
    Returns (head, flow, emitter); differentiable w.r.t. demand, res_head, ke,
    r_hw and the pump parameters speed / pump_h0 / pump_r ([L] or [B,L]; the
    reference takes these on its CPU adjoint only, dgga/autodiff.py:609-756).
    status (a frozen internal status) is refused: the batched status machine
    decides each scenario's status."""
    if adjoint == "cpu":
        raise NotImplementedError(
            "adjoint='cpu' is the reference's scipy splu adjoint; this package "
            "provides adjoint='gpu'")
    if adjoint != "gpu":
        raise ValueError("adjoint must be 'cpu'/'gpu', got %r" % (adjoint,))
    if status is not None:
        raise NotImplementedError(
            "adjoint='gpu' takes no status: the batched status machine decides "
            "each scenario's status")
    if assemble != "csr" or linear_solver != "sm100":
        raise ValueError("the B200 route is assemble='csr', linear_solver='sm100'")
    dev = solver.device
    t = lambda x: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    ke = solver.node_ke_default if ke is None else ke
    r_hw = solver.r_hw if r_hw is None else r_hw
    tn = lambda x: None if x is None else t(x)
    return ImplicitGGASolveSM100.apply(t(demand), t(res_head), t(ke), t(r_hw), solver,
                                       accuracy, max_iter, status_machine, int(polish_steps),
                                       tn(speed), tn(pump_h0), tn(pump_r))


class UnrolledSM100(torch.autograd.Function):
    """(demand, res_head, ke, r_hw, solver, K) -> (head[B,N], flow[B,L],
    emitter[B,N], relerr[B]): K GGA iterations with no convergence test and
    the initial statuses, differentiated through all of them
    (solve_unrolled, dgga/autodiff.py:1357-1664).  Forward: one wds_forward
    in unrolled mode, recording each iteration's state; backward: one
    wds_unrolled_adjoint (each iteration's factor rebuilt, one transposed
    solve per iteration).  1-D inputs get the batch-summed gradient."""

    @staticmethod
    def forward(ctx, demand, res_head, ke, r_hw, solver, K, warm=None):
        s = solver
        dims = (demand.dim(), res_head.dim(), ke.dim(), r_hw.dim())
        devs = (demand.device, res_head.device, ke.device, r_hw.device)
        d, rh, ke_t, r_t, B, _ = s._inputs(demand.detach(), res_head.detach(),
                                           ke.detach(), r_hw.detach())
        ke_t, r_t = ke_t.contiguous(), r_t.contiguous()
        rec = torch.empty(B, int(K), s.L + 2 * s.Nj, dtype=torch.float64, device=s.device)
        q0, e0, S0 = warm if warm is not None else (None, None, None)
        q0 = s._warm(q0, B, s.L)
        e0 = s._warm(e0, B, s.N)
        if S0 is not None:
            S0 = torch.as_tensor(np.asarray(S0), dtype=torch.int8, device=s.device)
            S0 = (S0.unsqueeze(0).expand(B, -1) if S0.dim() == 1 else S0).contiguous()
        o = s.run(d, rh, ke_t, r_t, B, int(K), 1e-12, False, -1, refine=2, refine_band=0.0,
                  record=rec, q0=q0, e0=e0, S0=S0)
        info = o["info"]
        if bool((info != 0).any()):
            from .solver import _check_info_flags
            _check_info_flags(s, info)
            bad = torch.nonzero(info != 0).flatten().tolist()
            raise RuntimeError("solve_unrolled: the node matrix of scenarios %s is not "
                               "positive definite%s" % (bad[:8], _not_pd_hint(s)))
        ctx.save_for_backward(d, rh, ke_t, r_t, rec)
        ctx.S0 = S0
        ctx.solver, ctx.plan, ctx.B, ctx.K, ctx.dims, ctx.devs = s, o["plan"], B, int(K), dims, devs
        head, flow, emit, relerr = o["head"], o["flow"], o["emit"], o["relerr"]
        if all(x == 1 for x in dims[:3]):
            head, flow, emit, relerr = head[0], flow[0], emit[0], relerr[0]
        ctx.mark_non_differentiable(relerr)
        return head, flow, emit, relerr

    @staticmethod
    def backward(ctx, gH, gQ, gE, _grel):
        if torch.is_grad_enabled():
            raise NotImplementedError("solve_unrolled on the sm100 route is first order only")
        s, p, B, K = ctx.solver, ctx.plan, ctx.B, ctx.K
        d, rh, ke_t, r_t, rec = ctx.saved_tensors
        dev, N, L = s.device, s.N, s.L

        def _g(g, n):
            if g is None:   # a read-only input of the adjoint: one cached zero block
                return s._zero_rows(B, n)
            g = g.detach().to(dtype=torch.float64, device=dev)
            return (g.unsqueeze(0).expand(B, -1) if g.dim() == 1 else g).contiguous()

        gH, gQ, gE = _g(gH, N), _g(gQ, L), _g(gE, N)
        gd = torch.empty(B, N, dtype=torch.float64, device=dev)
        grh, gke = torch.empty_like(gd), torch.empty_like(gd)
        gr = torch.empty(B, L, dtype=torch.float64, device=dev)
        scr = torch.empty(B, 2 * L + 2 * s.Nj, dtype=torch.float64, device=dev)
        cur = torch.cuda.current_stream(dev)
        _lib.check(p.lib.wds_unrolled_adjoint(
            p.handle, B, K, rec.data_ptr(), d.data_ptr(), rh.data_ptr(), ke_t.data_ptr(),
            0 if ke_t.shape[0] == 1 else N, r_t.data_ptr(), 0 if r_t.shape[0] == 1 else L,
            gH.data_ptr(), gQ.data_ptr(), gE.data_ptr(), gd.data_ptr(), grh.data_ptr(),
            gke.data_ptr(), gr.data_ptr(), scr.data_ptr(),
            None if ctx.S0 is None else ctx.S0.data_ptr(), ctypes.c_void_p(cur.cuda_stream)),
            "wds_unrolled_adjoint")
        dm, dv = ctx.dims, ctx.devs

        def _fit(g, dim, d_):
            g = g.to(device=d_)
            return g.sum(0) if dim == 1 else g

        return (_fit(gd, dm[0], dv[0]), _fit(grh, dm[1], dv[1]), _fit(gke, dm[2], dv[2]),
                _fit(gr, dm[3] + 1, dv[3]), None, None, None)


def solve_unrolled(solver, demand, res_head, ke=None, r_hw=None, K=None, q0=None, e0=None,
                   speed=None, status=None, pump_h0=None, pump_r=None, assemble="csr",
                   linear_solver="sm100"):
    """K fixed GGA iterations (no convergence test, statuses frozen: `status`,
    internal codes [L] or [B,L], or the initial ones), from the warm start
    q0 [L] or [B,L] / e0 [N] or [B,N] or the initial flows, differentiable
    w.r.t. demand, res_head, ke and r_hw through every iteration
    (dgga/autodiff.py:1357-1664 contract; the warm start is a constant, as
    an input without requires_grad in the reference).  Returns dict(head_ft,
    flow_cfs, emitter_cfs, relerr).  Like the reference: CVPIPE/PIPE/PUMP/TCV
    networks only (control valves refused), K defaults to the network's
    TRIALS.  Not taken on this route: pump parameters (speed, pump_h0,
    pump_r)."""
    if assemble != "csr" or linear_solver != "sm100":
        raise ValueError("the B200 route is assemble='csr', linear_solver='sm100'")
    if any(x is not None for x in (speed, pump_h0, pump_r)):
        raise NotImplementedError(
            "solve_unrolled on the sm100 route runs with the network's pump parameters "
            "(speed/pump_h0/pump_r refused; implicit_solve differentiates them)")
    s = solver
    lt = s._lt
    from .net import FCV as _FCV, PRV as _PRV, PSV as _PSV
    bad = np.flatnonzero(np.isin(lt, (_PRV, _PSV, _FCV)))
    if bad.size:
        raise NotImplementedError(
            "solve_unrolled supports CVPIPE/PIPE/PUMP/TCV; PRV/PSV/FCV (links %s) are not on "
            "the unrolled route - use implicit_solve" % bad[:8].tolist())
    dev = s.device
    t = lambda x: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    ke = s.node_ke_default if ke is None else ke
    r_hw = s.r_hw if r_hw is None else r_hw
    K = int(s.max_iter_default if K is None else K)
    det = lambda x: None if x is None else (x.detach() if isinstance(x, torch.Tensor) else x)
    if q0 is None and status is not None:
        # initlinkflow under the frozen statuses (dgga/autodiff.py:1472-1485):
        # closed links QZERO, the others as at set-up
        st = np.asarray(det(status).cpu() if isinstance(status, torch.Tensor) else status)
        q0 = np.where(st <= 2, 1e-6, s._q_open)
    warm = (det(q0), det(e0), det(status)) if any(x is not None for x in (q0, e0, status)) \
        else None
    head, flow, emit, relerr = UnrolledSM100.apply(t(demand), t(res_head), t(ke), t(r_hw), s, K,
                                                   warm)
    return dict(head_ft=head, flow_cfs=flow, emitter_cfs=emit, relerr=relerr)


# Thresholds and verdicts of the unrolled-gradient health probe
# (dgga/autodiff.py:1670-1760); the verdict strings are the reference's return
# values: usable, conditional (a search direction only), not advised.
GRAD_HEALTH_OK = 1e-8
GRAD_HEALTH_COND = 1e-5
VERDICT_OK, VERDICT_COND, VERDICT_NO = "\u53ef\u7528", "\u6709\u6761\u4ef6", "\u4e0d\u5efa\u8bae"


def unrolled_grad_health(solver, demand, res_head, ke=None, r_hw=None, K=None, dK=5,
                         param="demand", weights=None, vs_implicit=False, seed=0):
    """Per-network check that the unrolled gradient has settled in K
    (unrolled_grad_health, dgga/autodiff.py:1670-1760): the gradient of
    sum(weights * head) w.r.t. `param` at K + dK and at K + 2 dK, rel_K =
    max|g1 - g2| / max(|g1|, |g2|); with vs_implicit also against the implicit
    adjoint's gradient.  verdict: VERDICT_OK when rel_K < 1e-8 (and the
    implicit difference < 1e-6), VERDICT_COND when rel_K < 1e-5 (and < 1e-3),
    else VERDICT_NO (use implicit_solve).  K defaults to the forward's
    iteration count; weights to seeded normal values."""
    if param not in ("demand", "res_head", "ke", "r_hw"):
        raise ValueError("param must be demand/res_head/ke/r_hw, got %r" % (param,))
    s = solver
    dev = s.device
    t = lambda x: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    d0, rh0 = t(demand), t(res_head)
    ke0 = s.node_ke_default if ke is None else t(ke)
    r0 = s.r_hw if r_hw is None else t(r_hw)
    if K is None:
        with torch.no_grad():
            K = int(torch.as_tensor(s.solve(d0, rh0, ke_int=ke0,
                                            status_machine=bool(s.dense_status_machine))
                                    ["iters"]).max())
    K, dK = int(K), int(dK)
    B = d0.shape[0] if d0.dim() == 2 else 1
    if weights is None:
        g = np.random.default_rng(seed)
        shp = (B, s.N) if d0.dim() == 2 else (s.N,)
        weights = g.normal(0, 1, shp)
    W = t(weights)

    def _theta():
        th = dict(demand=d0.clone(), res_head=rh0.clone(), ke=ke0.clone(), r_hw=r0.clone())
        th[param].requires_grad_(True)
        return th

    def grad_at(kk):
        th = _theta()
        o = solve_unrolled(s, th["demand"], th["res_head"], ke=th["ke"], r_hw=th["r_hw"], K=kk)
        gg, = torch.autograd.grad((o["head_ft"] * W).sum(), th[param])
        return gg.detach()

    g1, g2 = grad_at(K + dK), grad_at(K + 2 * dK)
    den = float(torch.max(g1.abs().max(), g2.abs().max()).clamp_min(1e-300))
    rel_K = float((g1 - g2).abs().max()) / den
    rel_imp = None
    if vs_implicit:
        th = _theta()
        h = implicit_solve(s, th["demand"], th["res_head"], ke=th["ke"], r_hw=th["r_hw"],
                           accuracy=1e-10)[0]
        gi, = torch.autograd.grad((h * W).sum(), th[param])
        gi = gi.detach()
        dn = float(torch.max(g1.abs().max(), gi.abs().max()).clamp_min(1e-300))
        rel_imp = float((g1 - gi).abs().max()) / dn
    if rel_K < GRAD_HEALTH_OK and (rel_imp is None or rel_imp < 1e-6):
        verdict = VERDICT_OK
    elif rel_K < GRAD_HEALTH_COND and (rel_imp is None or rel_imp < 1e-3):
        verdict = VERDICT_COND
    else:
        verdict = VERDICT_NO
    return dict(verdict=verdict, rel_K=rel_K, rel_implicit=rel_imp, gmax=den, K=K, dK=dK,
                param=param)


# Roughness chain rule (dgga/calib.py:64-89): r = 4.727 L / C^1.852 / D^4.871.
def hw_resistance(C, length_ft, diam_ft):
    """Hazen-Williams resistance of pipes with roughness C (internal units)."""
    return 4.727 * length_ft / C ** 1.852 / diam_ft ** 4.871


def dr_dC(C, length_ft, diam_ft):
    """d r / d C = -1.852 r / C."""
    return -1.852 * hw_resistance(C, length_ft, diam_ft) / C
