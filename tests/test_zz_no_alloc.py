"""wds_forward_noalloc: the forward for callers that cannot allocate device
memory when they solve (a control loop that allocates everything at start-up
because an allocation can stall it, or a host process whose device memory
belongs to another allocator).  Its workspace is one fixed device array
shared by all calls instead of the plan's workspace; its results must be
those of wds_forward on the same inputs, bit for bit, call after call, with
whatever the previous call left in the array.

This file is collected last so that a run stopping at the first failure has
already run every other test."""
import ctypes

import numpy as np
import pytest
import torch

from wdsgpu_b200 import _lib, synth
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu

POLISHED_HEAD_ATOL_FT = 1e-9 / 0.3048   # the tolerance of the parity tests


def _outputs(B, N, L, dev):
    return dict(head=torch.empty(B, N, dtype=torch.float64, device=dev),
                flow=torch.empty(B, L, dtype=torch.float64, device=dev),
                emit=torch.empty(B, N, dtype=torch.float64, device=dev),
                status=torch.empty(B, L, dtype=torch.int8, device=dev),
                iters=torch.empty(B, dtype=torch.int32, device=dev),
                relerr=torch.empty(B, dtype=torch.float64, device=dev),
                info=torch.empty(B, dtype=torch.int32, device=dev))


def _noalloc(lib, plan, B, opts, d, rh, ke, r, out, stream):
    return lib.wds_forward_noalloc(
        plan.handle, B, ctypes.byref(opts), d.data_ptr(), rh.data_ptr(), ke.data_ptr(),
        r.data_ptr(), out["head"].data_ptr(), out["flow"].data_ptr(), out["emit"].data_ptr(),
        out["status"].data_ptr(), out["iters"].data_ptr(), out["relerr"].data_ptr(),
        out["info"].data_ptr(), ctypes.c_void_p(stream))


def _opts():
    opts = _lib.WdsForwardOpts()
    opts.accuracy, opts.max_iter, opts.status_machine = 1e-6, 200, 1
    opts.refine, opts.polish_steps, opts.ke_stride, opts.r_stride = 2, 3, 0, 0
    return opts


def _case(s, net, B, seed, cuda):
    d_np, rh_np = synth.config2_scenarios(net, B, seed=seed)
    d = torch.tensor(d_np, device=cuda)
    rh = torch.tensor(rh_np, device=cuda)
    ke = s.node_ke_default.unsqueeze(0).contiguous()
    r = s.r_hw.unsqueeze(0).contiguous()
    # wds_forward on the same inputs and options, in the plan's own workspace
    ref = s.run(d, rh, ke, r, B, 200, 1e-6, True, 3, refine=2, refine_band=0.0)
    return d, rh, ke, r, ref


def _check_calls(s, net, cuda, calls):
    """calls: (B, seed) per call, made in a row through wds_forward_noalloc;
    each must equal wds_forward on its inputs bitwise, whatever the earlier
    calls left in the shared array."""
    lib = _lib.load()
    opts = _opts()
    stream = torch.cuda.current_stream(cuda).cuda_stream
    for B, seed in calls:
        d, rh, ke, r, ref = _case(s, net, B, seed, cuda)
        torch.cuda.synchronize(cuda)
        out = _outputs(B, net.N, net.L, cuda)
        rc = _noalloc(lib, ref["plan"], B, opts, d, rh, ke, r, out, stream)
        assert rc == 0, lib.wds_last_error().decode()
        torch.cuda.synchronize(cuda)
        assert int(out["info"].abs().sum()) == 0
        for k in ("info", "iters", "status", "relerr", "head", "flow", "emit"):
            assert torch.equal(out[k], ref[k]), (B, seed, k)
        dh = float((out["head"] - ref["head"]).abs().max())
        assert dh <= POLISHED_HEAD_ATOL_FT


def test_noalloc_forward_matches_wds_forward_on_two_calls(cuda):
    # 3 PRVs: the polish uses the Woodbury scratch.  The first call runs other
    # scenarios at a larger batch, so the array holds other values (and more
    # of them) when the second call reads it.
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    _check_calls(s, net, cuda, [(96, 91), (48, 77)])


def test_noalloc_forward_large_network_layout(cuda):
    # the large-network layout keeps each scenario's whole state in the array
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    s.sm100_layout = "global"
    _check_calls(s, net, cuda, [(24, 93), (12, 78)])


def test_noalloc_rejects_a_batch_beyond_the_fixed_array(cuda):
    net = synth.config2_network()
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    p = s.plan(1)
    lib = _lib.load()
    B = 100000                                              # far beyond 64 MiB of workspace
    opts = _lib.WdsForwardOpts()
    opts.accuracy, opts.max_iter, opts.status_machine = 1e-6, 200, 1
    opts.refine, opts.polish_steps = 2, 3
    dummy = torch.zeros(1, dtype=torch.float64, device=cuda)
    rc = lib.wds_forward_noalloc(p.handle, B, ctypes.byref(opts), *([dummy.data_ptr()] * 11),
                                 ctypes.c_void_p(0))
    assert rc == -1
    msg = lib.wds_last_error().decode()
    assert "fixed array" in msg and "scenarios" in msg
