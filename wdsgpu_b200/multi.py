"""Networks of different sizes in one launch.

`implicit_solve_multi` takes one GGASolver per network and runs all of their
batches through a single `wds_forward_multi` launch (GGA with status machine,
polish and terminal factor per plan) and, in the backward pass, a single
`wds_adjoint_multi` launch.  Each network keeps its own plan: its schedule,
its layout (shared memory, or global memory for large networks) and its
scenario groups per CTA.  Per network the results are those of
`implicit_solve` (dgga/autodiff.py:1315-1351 contract); the reference has no
counterpart, its solver holds one network (dgga/solver.py:160).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .autodiff import _adjoint_guards, _clamp_grh, _clamp_rhs
from .solver import GGASolver, _Hold, _check_info_flags, _not_pd_hint

__all__ = ["implicit_solve_multi", "solve_multi"]


def _forward_multi(solvers, ins, accuracy, max_iter, status_machine, polish_steps):
    n = len(solvers)
    if not 1 <= n <= _lib.MULTI_MAX:
        raise ValueError("1 to %d networks per launch" % _lib.MULTI_MAX)
    if len({id(s) for s in solvers}) != n:
        raise ValueError("each network needs its own solver (a plan's workspace is per solver)")
    dev = solvers[0].device
    plans, outs = [], []
    opts = (_lib.WdsForwardOpts * n)()
    io = (_lib.WdsForwardIO * n)()
    batch = (ctypes.c_int32 * n)()
    for p, (s, (d, rh, ke, r, B)) in enumerate(zip(solvers, ins)):
        if s.device != dev:
            raise ValueError("all solvers must be on one device")
        pl = s.plan(B)
        plans.append(pl)
        o = dict(head=torch.empty(B, s.N, dtype=torch.float64, device=dev),
                 flow=torch.empty(B, s.L, dtype=torch.float64, device=dev),
                 emit=torch.empty(B, s.N, dtype=torch.float64, device=dev),
                 status=torch.empty(B, s.L, dtype=torch.int8, device=dev),
                 iters=torch.empty(B, dtype=torch.int32, device=dev),
                 relerr=torch.empty(B, dtype=torch.float64, device=dev),
                 info=torch.empty(B, dtype=torch.int32, device=dev), plan=pl,
                 _keep=(d, rh, ke, r))
        outs.append(o)
        op = opts[p]
        op.accuracy = float(accuracy)
        op.max_iter = int(max_iter)
        op.status_machine = 1 if status_machine else 0
        op.refine = s.refine_steps(accuracy)
        op.refine_band = s.refine_band(accuracy)
        op.polish_steps = int(polish_steps)
        op.ke_stride = 0 if ke.shape[0] == 1 else s.N
        op.r_stride = 0 if r.shape[0] == 1 else s.L
        x = io[p]
        x.demand, x.fixed_head, x.ke, x.r = d.data_ptr(), rh.data_ptr(), ke.data_ptr(), r.data_ptr()
        x.head, x.flow, x.emitter = o["head"].data_ptr(), o["flow"].data_ptr(), o["emit"].data_ptr()
        x.status, x.iters = o["status"].data_ptr(), o["iters"].data_ptr()
        x.relerr, x.info = o["relerr"].data_ptr(), o["info"].data_ptr()
        batch[p] = B
    handles = (ctypes.c_void_p * n)(*[pl.handle.value for pl in plans])
    cur = torch.cuda.current_stream(dev)
    _lib.check(plans[0].lib.wds_forward_multi(n, handles, batch, opts, io,
                                              ctypes.c_void_p(cur.cuda_stream)),
               "wds_forward_multi")
    return outs, plans


def _prep(solvers, demands, res_heads, kes, r_hws):
    ins = []
    for p, s in enumerate(solvers):
        ke = s.node_ke_default if kes is None or kes[p] is None else kes[p]
        r = s.r_hw if r_hws is None or r_hws[p] is None else r_hws[p]
        d, rh, ke_t, r_t, B, _ = s._inputs(demands[p], res_heads[p], ke, r)
        ins.append((d, rh, ke_t.contiguous(), r_t.contiguous(), B))
    return ins


def solve_multi(solvers, demands, res_heads, kes=None, r_hws=None, accuracy=None,
                max_iter=None, status_machine=True):
    """Steady GGA solve of several networks in one launch; per network the
    dict of GGASolver.solve (head_ft, flow_cfs, emitter_cfs, iters, relerr,
    converged[, status])."""
    s0 = solvers[0]
    acc = s0.hacc_default if accuracy is None else float(accuracy)
    mi = s0.max_iter_default if max_iter is None else int(max_iter)
    ins = _prep(solvers, demands, res_heads, kes, r_hws)
    outs, _ = _forward_multi(solvers, ins, acc, mi, status_machine, -1)
    res = []
    for s, o in zip(solvers, outs):
        info = o["info"]
        _check_info_flags(s, info)
        bad = torch.nonzero(info & _lib.INFO_NOT_PD).flatten()
        if bad.numel():
            raise RuntimeError("batched LDL^T failed: the node matrix of scenarios %s is not "
                               "positive definite%s" % (bad.tolist(), _not_pd_hint(s)))
        r = dict(head_ft=o["head"], flow_cfs=o["flow"], emitter_cfs=o["emit"],
                 iters=o["iters"].to(torch.int64), relerr=o["relerr"], converged=(info == 0))
        if status_machine:
            r["status"] = o["status"]
        res.append(r)
    return res


class ImplicitMultiSM100(torch.autograd.Function):
    """(n, solvers, accuracy, max_iter, polish_steps, then per network demand,
    res_head, ke, r_hw) -> per network (head, flow, emitter)."""

    @staticmethod
    def forward(ctx, n, solvers, accuracy, max_iter, polish_steps, *tensors):
        groups = [tensors[4 * p: 4 * p + 4] for p in range(n)]
        ins = []
        for s, (d, rh, ke, r) in zip(solvers, groups):
            d_, rh_, ke_, r_, B, _ = s._inputs(d.detach(), rh.detach(), ke.detach(), r.detach())
            ins.append((d_, rh_, ke_.contiguous(), r_.contiguous(), B))
        outs, plans = _forward_multi(solvers, ins, accuracy, max_iter, True, polish_steps)
        res, clamps = [], []
        for s, o in zip(solvers, outs):
            info = o["info"]
            _check_info_flags(s, info)
            if bool((info != 0).any()):
                bad = torch.nonzero(info != 0).flatten().tolist()
                if bool((info & _lib.INFO_NOT_PD).any()):
                    raise RuntimeError("implicit_solve_multi: the node matrix of scenarios %s "
                                       "is not positive definite%s" % (bad[:8], _not_pd_hint(s)))
                raise RuntimeError("implicit_solve_multi: scenarios %s did not converge"
                                   % bad[:8])
            clamps.append(_adjoint_guards(s, o["flow"], o["status"], allow_clamp=True))
            res += [o["head"], o["flow"], o["emit"]]
        ctx.solvers, ctx.plans, ctx.clamps = solvers, plans, clamps
        ctx.holds = [_Hold(pl) for pl in plans]   # kept until the backward
        ctx.B = [x[4] for x in ins]
        ctx.shapes = [(t.dim(), t.device) for t in tensors]
        return tuple(res)

    @staticmethod
    def backward(ctx, *grads):
        if torch.is_grad_enabled():
            raise NotImplementedError("implicit_solve_multi is first order only")
        solvers, plans = ctx.solvers, ctx.plans
        for h in ctx.holds:
            h.check("implicit_solve_multi backward")
        n = len(solvers)
        io = (_lib.WdsAdjointIO * n)()
        batch = (ctypes.c_int32 * n)()
        keep, outs, fixes = [], [], []
        for p, s in enumerate(solvers):
            B, dev = ctx.B[p], s.device

            def _g(g, cols):
                if g is None:
                    return torch.zeros(B, cols, dtype=torch.float64, device=dev)
                return g.detach().to(torch.float64).contiguous()

            gH, gQ, gE = _g(grads[3 * p], s.N), _g(grads[3 * p + 1], s.L), _g(grads[3 * p + 2], s.N)
            fix = None
            if ctx.clamps[p] is not None:   # constant-HP clamp branch: Woodbury, this plan
                gH, fix = _clamp_rhs(s, plans[p], B, ctx.clamps[p], gH, gQ, gE,
                                     torch.cuda.current_stream(dev).cuda_stream)
            fixes.append(fix)
            gd = torch.empty(B, s.N, dtype=torch.float64, device=dev)
            grh, gke = torch.empty_like(gd), torch.empty_like(gd)
            gr = torch.empty(B, s.L, dtype=torch.float64, device=dev)
            keep += [gH, gQ, gE]
            outs.append((gd, grh, gke, gr))
            x = io[p]
            x.gH, x.gQ, x.gE = gH.data_ptr(), gQ.data_ptr(), gE.data_ptr()
            x.gd, x.grh, x.gke, x.gr = gd.data_ptr(), grh.data_ptr(), gke.data_ptr(), gr.data_ptr()
            batch[p] = B
        handles = (ctypes.c_void_p * n)(*[pl.handle.value for pl in plans])
        cur = torch.cuda.current_stream(solvers[0].device)
        _lib.check(plans[0].lib.wds_adjoint_multi(n, handles, batch, io,
                                                  ctypes.c_void_p(cur.cuda_stream)),
                   "wds_adjoint_multi")
        for h in ctx.holds:
            h.release()
        for p in range(n):
            if fixes[p] is not None:
                _clamp_grh(fixes[p], keep[3 * p + 1], outs[p][0], outs[p][1])
        # [B, *] gradients; autograd sums them to a 1-D or single-row input's
        # shape (the batch sum of dgga/autodiff.py:1306-1308)
        res = []
        for p in range(n):
            for q, g in enumerate(outs[p]):
                res.append(g.to(device=ctx.shapes[4 * p + q][1]))
        return (None, None, None, None, None, *res)


def implicit_solve_multi(solvers, demands, res_heads, kes=None, r_hws=None, accuracy=1e-12,
                         max_iter=200, polish_steps=3):
    """Forward + implicit adjoint of several networks (one solver each) in one
    launch per pass.  Returns a list of (head, flow, emitter), differentiable
    w.r.t. each network's demand, res_head, ke and r_hw."""
    t = lambda x, dev: x.to(dtype=torch.float64, device=dev) if isinstance(x, torch.Tensor) \
        else torch.as_tensor(np.asarray(x), dtype=torch.float64, device=dev)
    flat = []
    for p, s in enumerate(solvers):
        dev = s.device
        ke = s.node_ke_default if kes is None or kes[p] is None else kes[p]
        r = s.r_hw if r_hws is None or r_hws[p] is None else r_hws[p]
        flat += [t(demands[p], dev), t(res_heads[p], dev), t(ke, dev), t(r, dev)]
    out = ImplicitMultiSM100.apply(len(solvers), list(solvers), float(accuracy), int(max_iter),
                                   int(polish_steps), *flat)
    return [tuple(out[3 * p: 3 * p + 3]) for p in range(len(solvers))]
