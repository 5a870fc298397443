"""The measured autotuner (wdsgpu_b200.tune): it times the planner's schedule
choices, keeps the cost model's choice unless a measured one is faster, and
caches the result; a tuned plan gives the default plan's results within
rounding (iterations and statuses equal, polished heads within 1e-9 m,
gradients within 1e-9 relative)."""
import json

import numpy as np
import pytest
import torch

from tests.golden.load import load
from wdsgpu_b200 import tune
from wdsgpu_b200.autodiff import implicit_solve
from wdsgpu_b200.solver import GGASolver

pytestmark = pytest.mark.gpu


def _step(s, d, rh, sens, cuda):
    D = torch.tensor(d, device=cuda, requires_grad=True)
    o = s.solve(torch.tensor(d, device=cuda), torch.tensor(rh, device=cuda), accuracy=1e-6,
                status_machine=True)
    h = implicit_solve(s, D, torch.tensor(rh, device=cuda), accuracy=1e-6)[0]
    (h[:, sens] ** 2).sum().backward()
    return o, h.detach().cpu().numpy(), D.grad.cpu().numpy()


@pytest.mark.parametrize("tag", ["cfg3_small", "cfg2"])
def test_autotune_keeps_results_and_caches(cuda, tmp_path, tag):
    net, inp, _ = load(tag)
    B = 64
    rng = np.random.default_rng(6)
    d = np.repeat(inp["demand"][:1], B, 0) * rng.lognormal(0.0, 0.2, (B, net.N))
    rh = np.repeat(np.nan_to_num(inp["res_head"][:1]), B, 0)
    sens = np.asarray(inp["sensors"])
    cache = str(tmp_path / "tune.json")
    s = GGASolver(net, device=cuda, dense_status_machine=True)
    res = tune.autotune(s, B, d, rh, repeats=1, cache_path=cache)
    assert res["ms"] <= res["model_ms"]
    assert len(res["tried"]) >= 3
    assert json.load(open(cache))[res["key"]]["choice"] == res["choice"]
    ref = GGASolver(net, device=cuda, dense_status_machine=True)
    o0, h0, g0 = _step(ref, d, rh, sens, cuda)
    for choice in [res["choice"], {"groups_per_cta": 1, "top_max": 16,
                                   "level_barrier_cost": 8.0}]:
        s2 = GGASolver(net, device=cuda, dense_status_machine=True)
        s2.sm100_tuning = choice
        o1, h1, g1 = _step(s2, d, rh, sens, cuda)
        assert torch.equal(o0["iters"], o1["iters"]) and torch.equal(o0["status"], o1["status"])
        assert np.abs(h1 - h0).max() <= 1e-9 / 0.3048
        assert np.abs(g1 - g0).max() <= 1e-9 * np.abs(g0).max()
    s3 = GGASolver(net, device=cuda, dense_status_machine=True)
    assert tune.apply_cached(s3, B, cache_path=cache) == res["choice"]
    assert s3.sm100_tuning == (res["choice"] or None)
