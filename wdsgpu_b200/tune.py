"""Measured autotuner of the planner's schedule choices.

The planner (`wds_plan`) picks, from a cost model over the network's
symbolic structure, the scenario groups per CTA, the size of the dense top
block and, per elimination-tree level, the lane-group size and whether the
level runs on the whole group or on one warp.  `autotune` replaces those
guesses by measurements on the GPU at hand: it times one forward + implicit
adjoint step (`implicit_solve` and the backward of a sum of squared heads)
for a few values of each choice, by coordinate search from the cost model's
choice, keeps the fastest whose polished heads agree with the cost model's
plan, and stores the choice in a JSON cache keyed by the network's tables,
the batch size and the device name, so that a later process applies it
without timing (`apply_cached`).

The choices change the schedule, not the algorithm: a tuned plan's results
agree with the default plan's within rounding (the order of a few dot
products and of the dense top block's inverse differ), iteration counts and
statuses included on the parity workloads.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import torch

__all__ = ["autotune", "apply_cached", "network_key", "default_cache_path"]

# values tried for each choice, in the order of the coordinate search
GROUPS = (1, 2, 3, 4)
TOP_MAX = (32, 16, -1)
BARRIER_COST = (0.25, 2.0, 8.0)


def default_cache_path():
    """WDSGPU_B200_TUNE_CACHE, else ~/.cache/wdsgpu_b200/tune.json."""
    return os.environ.get("WDSGPU_B200_TUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "wdsgpu_b200", "tune.json")


def network_key(solver, batch):
    """Hash of the tables the planner sees, the batch size and the device."""
    h = hashlib.sha256()
    for k in sorted(solver._tables):
        a = np.ascontiguousarray(solver._tables[k])
        h.update(k.encode())
        h.update(a.tobytes())
    h.update(str(int(batch)).encode())
    h.update(torch.cuda.get_device_name(solver.device).encode())
    h.update(str(solver.sm100_factor_dtype).encode())
    return h.hexdigest()[:32]


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, key, entry):
    data = _load(path)
    data[key] = entry
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def _reset_plans(solver, tuning):
    for p in solver._plans:
        p.free()
    solver._plans = []
    solver.sm100_tuning = tuning


def _time_step(solver, demand, res_head, sens, accuracy, repeats):
    """Median device time (ms) of one forward + adjoint step and its heads."""
    from .autodiff import implicit_solve
    dev = solver.device
    times, heads = [], None
    for i in range(repeats + 1):
        D = demand.clone().requires_grad_(True)
        torch.cuda.synchronize(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        h = implicit_solve(solver, D, res_head, accuracy=accuracy, status_machine=True)[0]
        (h.index_select(1, sens) ** 2).sum().backward()
        e1.record()
        torch.cuda.synchronize(dev)
        if i > 0:                       # the first run builds the plan
            times.append(e0.elapsed_time(e1))
        heads = h.detach()
    return float(np.median(times)), heads


def autotune(solver, batch, demand=None, res_head=None, accuracy=1e-6, repeats=3,
             cache_path=None, n_sensors=30, head_atol_ft=1e-7, margin=0.98):
    """Time the candidate schedule choices for `batch` scenarios and set the
    fastest on `solver` (its plans are rebuilt).  demand / res_head [B,N]
    default to the network's base demand with lognormal(0.2) factors and its
    reservoir heads.  A choice replaces the current best only when it is
    faster by more than 1 - margin.  Returns dict(choice, ms, model_ms, key,
    tried)."""
    from . import synth
    dev = solver.device
    net = solver.net
    B = int(batch)
    if demand is None or res_head is None:
        d, rh = synth.config2_scenarios(net, B, seed=12345)
        demand = d if demand is None else demand
        res_head = np.nan_to_num(rh) if res_head is None else res_head
    demand = torch.as_tensor(np.asarray(demand), dtype=torch.float64, device=dev)
    res_head = torch.as_tensor(np.asarray(res_head), dtype=torch.float64, device=dev)
    sens = torch.as_tensor(synth.sensor_nodes(net, min(n_sensors, solver.Nj)), device=dev)
    _reset_plans(solver, None)
    model_ms, ref_heads = _time_step(solver, demand, res_head, sens, accuracy, repeats)
    best, best_ms = {}, model_ms
    tried = [({}, model_ms)]

    def attempt(choice):
        try:
            _reset_plans(solver, choice)
            ms, h = _time_step(solver, demand, res_head, sens, accuracy, repeats)
        except (ValueError, NotImplementedError, RuntimeError):
            return None                 # does not fit, or refused on this network
        if float((h - ref_heads).abs().max()) > head_atol_ft:
            return None
        tried.append((dict(choice), ms))
        return ms

    for name, values in (("groups_per_cta", GROUPS), ("top_max", TOP_MAX),
                         ("level_barrier_cost", BARRIER_COST)):
        for v in values:
            choice = dict(best)
            choice[name] = v
            ms = attempt(choice)
            if ms is not None and ms < margin * best_ms:   # faster beyond timing noise
                best, best_ms = choice, ms
    _reset_plans(solver, best or None)
    key = network_key(solver, B)
    entry = dict(choice=best, ms=best_ms, model_ms=model_ms)
    _store(cache_path or default_cache_path(), key, entry)
    return dict(choice=best, ms=best_ms, model_ms=model_ms, key=key,
                tried=[dict(choice=c, ms=m) for c, m in tried])


def apply_cached(solver, batch, cache_path=None):
    """Set the cached choice for this network, batch and device on `solver`;
    returns it, or None when nothing is cached (the cost model stays)."""
    entry = _load(cache_path or default_cache_path()).get(network_key(solver, batch))
    if entry is None:
        return None
    _reset_plans(solver, entry["choice"] or None)
    return entry["choice"]
