"""Benchmark: forward + implicit adjoint scenarios/s at B=1024 on the
782-junction synthetic network (905 pipes, 3 PRVs, 2 reservoirs, 20 emitters).

One step = one pass of the hot path over one batch: the batched GGA solve
with the status machine, the 3-step reduced Newton polish, the terminal
factorisation, the implicit adjoint of loss = sum of squared heads at 30
sensor junctions, and the gradients w.r.t. demand, pipe roughness (chain rule
through r = 4.727 L / C^1.852 / D^4.871) and emitter coefficients.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sm100|reference]
    python bench.py --workload mixed|eps      (secondary workloads, one GPU)

`--workload mixed`: 256 instances drawn uniformly from four networks (100,
542 with 79 TCVs, 782 with 3 PRVs, 3000 junctions), forward + adjoint in one
multi-plan launch per pass.  `--workload eps`: 24 hourly steps of the
20 000-junction pump/tank network, B=64, forward + adjoint through time.

N > 1 is launched with torch.distributed.run: every rank solves its own
batch of 1024 scenarios (weak scaling); the batch-summed roughness and
emitter gradients are all-reduced over NCCL.  Rank 0 prints one JSON line.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fwd+adjoint scenarios/s at B=1024 (782 jn) vs ref cuDSS on B200, at 1e-9 m head err"
UNIT = "scenarios/s"
WORKLOAD = ("782-junction synthetic looped network (905 pipes, 3 PRVs, 2 reservoirs, "
            "20 emitters), B=1024 lognormal(0.2) demand scenarios; batched GGA with "
            "status machine (accuracy 1e-6) + 3-step Newton polish + implicit adjoint of "
            "sum of squared heads at 30 sensors; grads w.r.t. demand, roughness C, emitter Ke")
N_SENSORS = 30
POLISH = 3
ACCURACY = 1e-6


def bytes_per_iteration(L, nA, nL, Nj, w=8, refine=2):
    """Streaming model of one Newton iteration: coefficients 24 L, assembly
    8 L + 8 nA + 8 Nj, LDL^T w (nA + nL), solve 2 w nL + 16 Nj, each
    refinement 8 nA + 2 w nL + 32 Nj, update 8 Nj + 32 L; with 2 refinements
    64 L + (24 + w) nA + 7 w nL + 96 Nj."""
    return (64 * L + (8 + w + 8 * refine) * nA + (3 + 2 * refine) * w * nL
            + (32 + 32 * refine) * Nj)


def adjoint_bytes(L, N, nA, nL, Nj, w=8):
    """RHS, one solve + 2 refinements on the kept factor, gradient writes."""
    return 24 * L + (6 * w * nL + 16 * nA + 80 * Nj) + 8 * (2 * N + L)


def read_profile_traffic():
    """Per-scenario DRAM bytes of the forward kernel from the committed ncu
    summary (None when absent)."""
    p = os.path.join(ROOT, "profiles", "k_forward_config2.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_scenario:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            cmd = ["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                   "-lms", "100"]
            if self.gpu_id is not None:
                cmd += ["-i", str(self.gpu_id)]
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
            time.sleep(0.3)   # nvidia-smi's first sample before the timed region starts
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        return False

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _gpu_id_for(dev_index):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        if dev_index < len(ids):
            return ids[dev_index]
    return dev_index


# ------------------------------------------------------------------ CPU legs
def _oracle_scenarios(payload):
    """Oracle fwd + polish + adjoint on a few scenarios (one process)."""
    import numpy as np
    from threadpoolctl import threadpool_limits
    sys.path.insert(0, ROOT)
    from oracle.gga import Model
    from wdsgpu_b200 import synth
    d, rh = payload
    with threadpool_limits(1):
        net = synth.config2_network()
        m = Model(net)
        sens = synth.sensor_nodes(net, N_SENSORS)
        out, st = m.implicit(d, rh, accuracy=ACCURACY, polish_steps=POLISH)
        gH = np.zeros_like(out["head_ft"])
        gH[:, sens] = 2.0 * out["head_ft"][:, sens]
        g = m.backward(st, gH, np.zeros_like(out["flow_cfs"]), np.zeros_like(out["emitter_cfs"]))
    return float(g[0].sum())


def cpu_baseline_single(n_scen=36):
    """The oracle port timed on one host core (the `cpu_baseline` object), on
    a sample of about ten seconds of CPU work."""
    from wdsgpu_b200 import synth
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, n_scen, seed=4242)
    t0 = time.perf_counter()
    _oracle_scenarios((d, rh))
    dt = time.perf_counter() - t0
    return {"value": n_scen / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "%d scenarios of the B=1024 workload (fwd + 3-step polish + adjoint), "
                      "numpy oracle, one core, %.1f s" % (n_scen, dt)}


def run_reference(args, rank, world):
    """`--impl reference`: the reference algorithm's CPU restatement (the
    oracle port) on every host core, one scenario per worker per step."""
    if rank != 0:
        return
    import multiprocessing as mp
    from wdsgpu_b200 import synth
    cores = physical_cores()            # SMT siblings counted once
    workers = max(1, min(cores, 32))
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 1024, seed=1000)
    ctx = mp.get_context("spawn")
    times = []
    # each step is one scenario per worker (about a second of CPU work); at
    # most 10 steps are timed so that the arm ends within a few minutes
    n_steps = min(args.steps, 10)
    with ctx.Pool(workers) as pool:
        k = 0
        for i in range(min(args.warmup, 3) + n_steps):
            chunks = []
            for _ in range(workers):
                chunks.append((d[k % 1024:k % 1024 + 1], rh[k % 1024:k % 1024 + 1]))
                k += 1
            t0 = time.perf_counter()
            pool.map(_oracle_scenarios, chunks)
            if i >= min(args.warmup, 3):
                times.append(time.perf_counter() - t0)
    ms = 1e3 * statistics.mean(times)
    value = workers / (ms / 1e3)
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": n_steps, "warmup": min(args.warmup, 3), "steps_requested": args.steps,
            "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": WORKLOAD, "B": 1024, "sample_per_step": workers},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": "port",
                             "sample": "%d scenarios per step (one per worker process, "
                                       "numpy oracle restating the reference dense route)"
                                       % workers},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ the reference's own code
def _reference_package():
    """The unmodified reference (package `dgga`) installed offline into
    baseline/_ref.  Its INP parser imports `wntr` at module top, which is not
    installed; a stub with the imported names stands in (the parser is never
    called: the network is built here and handed over as a `Net`)."""
    import types
    ref = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(ref, "dgga")):
        return None, "reference not installed in baseline/_ref"
    if "wntr" not in sys.modules:
        w = types.ModuleType("wntr")
        ep = types.ModuleType("wntr.epanet")
        ut = types.ModuleType("wntr.epanet.util")
        ut.FlowUnits = type("FlowUnits", (), {})
        nw = types.ModuleType("wntr.network")
        el = types.ModuleType("wntr.network.elements")
        for n in ("Junction", "Reservoir", "Tank", "Pipe", "Pump", "Valve"):
            setattr(el, n, type(n, (), {}))
        w.epanet, ep.util, w.network, nw.elements = ep, ut, nw, el
        sys.modules.update({"wntr": w, "wntr.epanet": ep, "wntr.epanet.util": ut,
                            "wntr.network": nw, "wntr.network.elements": el})
    sys.path.insert(0, ref)
    import dgga.autodiff
    import dgga.parse
    import dgga.solver
    return dgga, None


def physical_cores():
    """Physical cores of this host (SMT siblings counted once)."""
    try:
        seen = set()
        base = "/sys/devices/system/cpu"
        for c in os.listdir(base):
            f = os.path.join(base, c, "topology", "core_id")
            g = os.path.join(base, c, "topology", "physical_package_id")
            if c.startswith("cpu") and c[3:].isdigit() and os.path.exists(f):
                seen.add((open(g).read().strip(), open(f).read().strip()))
        if seen:
            return len(seen)
    except OSError:
        pass
    return os.cpu_count() or 1


def run_reference_code(args):
    """`--workload refgpu|refcpu`: the reference's own implementation of the
    path, unmodified, through its public API (dgga/autodiff.py:1315-1351), on
    the bench workload: GGASolver(mode="dense", dense_status_machine=True) and
    implicit_solve(..., adjoint="gpu", accuracy=1e-6, status_machine=True),
    the loss and gradients of the bench step.  refgpu: its GPU route on this
    B200 at the full B (dense route: torch batched Cholesky; the cuDSS route
    when nvmath is importable), device time per step with CUDA events around
    the call, best-of and median as in scripts/mainline_v2/mv2_time_gpu.py:
    72-87.  refcpu: the same route on the host cores (torch threads = physical
    cores) on a sample of scenarios per step."""
    import torch
    from wdsgpu_b200 import synth
    dgga, why = _reference_package()
    gpu = args.workload == "refgpu"
    if dgga is None:
        print(json.dumps({"impl": "reference-code", "workload": args.workload,
                          "unavailable": why}), flush=True)
        return
    try:
        import nvmath  # noqa: F401
        have_cudss = gpu
    except ImportError:
        have_cudss = False
    cores = physical_cores()
    if gpu:
        dev = torch.device("cuda", 0)
        torch.cuda.set_device(dev)
        B = args.batch
    else:
        dev = torch.device("cpu")
        torch.set_num_threads(cores)
        B = 16
    net = synth.config2_network()
    rnet = dgga.parse.Net(**net.as_fields())
    s = dgga.solver.GGASolver(rnet, device=str(dev), dtype=torch.float64, mode="dense",
                              dense_status_machine=True)
    d_np, rh_np = synth.config2_scenarios(net, B, seed=1000)
    sens = torch.as_tensor(synth.sensor_nodes(net, N_SENSORS), device=dev)
    D0 = torch.as_tensor(d_np, device=dev)
    RH = torch.as_tensor(rh_np, device=dev)
    R0 = torch.as_tensor(np.asarray(net.r_hw), device=dev)
    K0 = torch.as_tensor(np.asarray(net.node_ke), device=dev)
    routes = [("dense", "dense")] + ([("csr", "cudss")] if have_cudss else [])
    res = {}
    for asm, ls in routes:
        def step():
            D = D0.clone().requires_grad_(True)
            R = R0.clone().requires_grad_(True)
            K = K0.clone().requires_grad_(True)
            h, q, e = dgga.autodiff.implicit_solve(
                s, D, RH, ke=K, r_hw=R, accuracy=ACCURACY, max_iter=200,
                polish_steps=POLISH, adjoint="gpu", status_machine=True, assemble=asm,
                linear_solver=ls)
            (h.index_select(1, sens) ** 2).sum().backward()
            return D.grad

        ms = []
        for i in range(max(1, args.warmup) + args.steps):
            if gpu:
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                step()
                e1.record()
                torch.cuda.synchronize()
                t = e0.elapsed_time(e1)
            else:
                t0 = time.perf_counter()
                step()
                t = 1e3 * (time.perf_counter() - t0)
            if i >= max(1, args.warmup):
                ms.append(t)
        res[ls] = {"best_ms": min(ms), "median_ms": statistics.median(ms),
                   "scenarios_per_s_best": B / (min(ms) / 1e3),
                   "scenarios_per_s_median": B / (statistics.median(ms) / 1e3)}
    main_route = "cudss" if "cudss" in res else "dense"
    value = res[main_route]["scenarios_per_s_median"]
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1 if gpu else 0,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": res[main_route]["median_ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference-code", "workload": args.workload,
            "config": {"workload": WORKLOAD.replace("B=1024", "B=%d" % B), "B": B,
                       "route": "%s/%s" % ("csr" if main_route == "cudss" else "dense",
                                           main_route),
                       "cudss": "available" if have_cudss else
                                "unavailable on this box (nvmath not installed)",
                       "device": torch.cuda.get_device_name(0) if gpu else "host cpu",
                       "torch_threads": None if gpu else cores},
            "routes": res}
    print(json.dumps(line), flush=True)


def run_tune(args):
    """`--workload tune`: the measured autotuner (wdsgpu_b200.tune) on the
    four networks of the mixed-size workload, each at `--batch` scenarios
    (default 256): the cost model's forward + adjoint step time beside the
    tuned one, and the choice.  One JSON line."""
    import tempfile
    import torch
    from wdsgpu_b200 import synth, tune
    from wdsgpu_b200.solver import GGASolver
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    B = 256 if args.batch == 1024 else args.batch
    names = ("100 jn / 120 pipes", "542 jn / 554 links, 79 TCVs", "782 jn / 905 pipes / 3 PRVs",
             "3000 jn / 3600 pipes")
    cache = os.path.join(tempfile.mkdtemp(), "tune.json")
    res = {}
    with ClockSampler(None) as clk:
        for name, net in zip(names, synth.config3_networks()):
            s = GGASolver(net, device=dev, dense_status_machine=True)
            r = tune.autotune(s, B, repeats=max(3, args.steps), cache_path=cache)
            res[name] = {"model_ms": r["model_ms"], "tuned_ms": r["ms"], "choice": r["choice"],
                         "candidates": len(r["tried"])}
    tot_m = sum(v["model_ms"] for v in res.values())
    tot_t = sum(v["tuned_ms"] for v in res.values())
    line = {"metric": "autotuned fwd+adjoint step time over the mixed-size networks "
                      "(sum of the four, B=%d each)" % B,
            "value": tot_t, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": tot_t, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "config-3 networks, one solver each, B=%d lognormal(0.2) "
                                   "scenarios; median of the timed steps per candidate" % B},
            "cost_model_ms": tot_m, "networks": res, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ secondary workloads
def run_secondary(args):
    """Mixed-size one-launch, extended-period and unrolled-K workloads: one JSON line."""
    import torch
    from wdsgpu_b200 import synth
    from wdsgpu_b200.solver import GGASolver
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    if args.workload == "mixed":
        from wdsgpu_b200.multi import implicit_solve_multi
        nets = synth.config3_networks()
        counts = np.bincount(np.random.default_rng(3).integers(0, 4, 256), minlength=4)
        solvers = [GGASolver(n, device=dev, dense_status_machine=True) for n in nets]
        data = []
        for i, (n, c) in enumerate(zip(nets, counts)):
            d, _ = synth.config2_scenarios(n, int(c), seed=50 + i, sigma=0.3)
            rh = np.broadcast_to(np.nan_to_num(n.fixed_head_ft_at(0)), d.shape).copy()
            data.append((torch.as_tensor(d, device=dev), torch.as_tensor(rh, device=dev)))
        sens = [torch.as_tensor(synth.sensor_nodes(n, 8), device=dev) for n in nets]

        def step():
            Ds = [d.clone().requires_grad_(True) for d, _ in data]
            outs = implicit_solve_multi(solvers, Ds, [rh for _, rh in data], accuracy=ACCURACY)
            loss = sum((h[:, sv] ** 2).sum() for (h, _, _), sv in zip(outs, sens))
            loss.backward()
            return sum(float(D.grad.abs().sum()) for D in Ds)

        units = int(counts.sum())
        metric = ("mixed-size fwd+adjoint instances/s (256 instances of 100/542/782/3000-junction "
                  "networks, one multi-plan launch per pass)")
        unit = "instances/s"
        cfg = {"workload": "mixed-size: networks of 100 jn/120 pipes, 542 jn/554 links with 79 TCVs, "
                           "782 jn/905 pipes/3 PRVs, 3000 jn/3600 pipes; instances per network %s; "
                           "lognormal(0.3) demands" % counts.tolist(),
               "instances": units, "launches_per_step": 2}
    elif args.workload == "unrolled":
        from wdsgpu_b200.autodiff import solve_unrolled
        from wdsgpu_b200.net import PIPE, PRV
        base = synth.config2_network()
        f = base.as_fields()                     # the unrolled route takes no PRVs
        lt = np.asarray(base.link_type).copy()
        st = np.asarray(base.init_status).copy()
        st[lt == PRV] = 1
        lt[lt == PRV] = PIPE
        f["link_type"], f["init_status"] = lt.astype(np.int8), st.astype(np.int8)
        net = synth.Net(**f)
        s = GGASolver(net, device=dev, dense_status_machine=True)
        B, K = 1024, 14
        d, rh = synth.config2_scenarios(net, B, seed=7)
        d = torch.as_tensor(d, device=dev)
        rh = torch.as_tensor(rh, device=dev)
        sens = torch.as_tensor(synth.sensor_nodes(net, N_SENSORS), device=dev)

        def step():
            D = d.clone().requires_grad_(True)
            out = solve_unrolled(s, D, rh, K=K)
            (out["head_ft"][:, sens] ** 2).sum().backward()
            return float(D.grad.abs().sum())

        units = B
        metric = "unrolled-K fwd+reverse scenarios/s (782 jn, K=14, B=1024)"
        unit = "scenarios/s"
        cfg = {"workload": "782-junction synthetic looped network with its 3 PRVs as open "
                           "pipes (the unrolled route takes no control valves); B=1024 "
                           "lognormal(0.2) demands; K=14 fixed GGA iterations recorded, then "
                           "the reverse pass over them (one factor and one solve per "
                           "iteration); grads w.r.t. demand of sum of squared heads at 30 "
                           "sensors", "B": B, "K": K}
    else:
        from wdsgpu_b200.eps import eps_solve
        net0 = synth.config5_network()
        pre = synth.tanks_as_junctions(net0)
        s0 = GGASolver(pre, device=dev, dense_status_machine=True)
        o = s0.solve(pre.demand_cfs_at(0)[None] * synth.diurnal(0.0),
                     np.nan_to_num(pre.fixed_head_ft_at(0))[None], status_machine=True,
                     accuracy=1e-8)
        ctr = o["head_ft"][0].cpu().numpy()[np.asarray(net0.tank_node)]
        net = synth.config5_network(tank_center_ft=ctr)
        s = GGASolver(net, device=dev, dense_status_machine=True)
        B, T = 64, 24
        dem = torch.as_tensor(synth.eps_demands(net, T, B, seed=6), device=dev)
        sens = torch.arange(0, net.N, 200, device=dev)

        frames = []

        def step():
            D = dem.clone().requires_grad_(True)
            out = eps_solve(s, D, accuracy=ACCURACY)
            loss = (out["head"][:, :, sens] ** 2).sum() + (out["tank_head"][-1] ** 2).sum()
            loss.backward()
            frames.append(int(out["valid"].sum()))
            return float(D.grad.abs().sum())

        step()
        units = frames[-1]
        metric = ("EPS fwd+adjoint scenario-frames/s (20 000 jn, 24 hourly demand periods, "
                  "B=64, EpsDriver's clock)")
        unit = "scenario-frames/s"
        cfg = {"workload": "extended period: about 20 000 junctions / 23 000 pipes, 4 pumps, "
                           "3 tanks, 1 reservoir; 24 hourly demand periods (23 h), frames on "
                           "EpsDriver's clock (steps shortened at tank fill/empty times), "
                           "statuses carried; B=64 diurnal x lognormal(0.15) demands; adjoint "
                           "through time with per-frame recomputation",
               "B": B, "frames_per_run": units, "layout": "global (large network)"}
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(None) as clk:
        for _ in range(args.steps):
            flush.fill_(1.0)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            step()
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1))
    ms = sum(times) / len(times)
    cfg["l2"] = "flushed between steps (256 MB write, outside the timed events)"
    line = {"metric": metric, "value": units / (ms / 1000.0), "unit": unit, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def fp32_form(net, d_dev, rh_dev, sens, B):
    """The same step with the FP32 factor and FP64 refinement
    (sm100_factor_dtype = float32): its time per step and its head and
    gradient differences from the FP64 form, or the refusal it raises."""
    import torch
    from wdsgpu_b200.autodiff import implicit_solve
    from wdsgpu_b200.solver import GGASolver
    out = {}
    for name, dt in (("fp64", torch.float64), ("fp32", torch.float32)):
        s = GGASolver(net, device=d_dev.device, dense_status_machine=True)
        s.sm100_factor_dtype = dt
        try:
            D = d_dev.clone().requires_grad_(True)
            h = implicit_solve(s, D, rh_dev, accuracy=ACCURACY, polish_steps=POLISH,
                               status_machine=True)[0]
            (h.index_select(1, sens) ** 2).sum().backward()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            D2 = d_dev.clone().requires_grad_(True)
            h2 = implicit_solve(s, D2, rh_dev, accuracy=ACCURACY, polish_steps=POLISH,
                                status_machine=True)[0]
            (h2.index_select(1, sens) ** 2).sum().backward()
            e1.record()
            torch.cuda.synchronize()
            out[name] = {"ms": e0.elapsed_time(e1), "head": h2.detach(), "grad": D2.grad}
        except RuntimeError as exc:
            out[name] = {"refused": str(exc)[:200]}
    res = {"fp64_scenarios_per_s": B / (out["fp64"]["ms"] / 1e3)}
    if "refused" in out["fp32"]:
        res["fp32"] = "refused: " + out["fp32"]["refused"]
    else:
        g64, g32 = out["fp64"]["grad"], out["fp32"]["grad"]
        res.update({"fp32_scenarios_per_s": B / (out["fp32"]["ms"] / 1e3),
                    "max_head_diff_m": float((out["fp32"]["head"] - out["fp64"]["head"])
                                             .abs().max()) * 0.3048,
                    "grad_rel_diff": float((g32 - g64).abs().max() / g64.abs().max())})
    return res


# ------------------------------------------------------------------ GPU leg
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="sm100", choices=("sm100", "reference"))
    ap.add_argument("--batch", type=int, default=1024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="config2",
                    choices=("config2", "config4", "mixed", "eps", "unrolled", "refgpu", "refcpu",
                             "tune"))
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.workload in ("refgpu", "refcpu"):
        run_reference_code(args)
        return
    if args.workload == "tune":
        run_tune(args)
        return
    if args.workload == "config4":
        args.batch = 16384 if args.batch == 1024 else args.batch
    elif args.workload != "config2":
        run_secondary(args)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from wdsgpu_b200 import synth
    from wdsgpu_b200.autodiff import dr_dC, implicit_solve
    from wdsgpu_b200.sharding import allreduce_batch_summed
    from wdsgpu_b200.solver import GGASolver

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    B = args.batch
    net = synth.config2_network()
    s = GGASolver(net, device=dev, dense_status_machine=True)
    d_np, rh_np = synth.config2_scenarios(net, B, seed=1000 + rank)
    sens = torch.as_tensor(synth.sensor_nodes(net, N_SENSORS), device=dev)
    C = torch.as_tensor(np.asarray(net.roughness), device=dev)
    length = torch.as_tensor(np.asarray(net.len_ft), device=dev)
    diam = torch.as_tensor(np.asarray(net.diam_ft), device=dev)
    is_pipe = torch.as_tensor(np.asarray(net.link_type) == 1, device=dev)
    dC = torch.where(is_pipe, dr_dC(torch.where(is_pipe, C, torch.ones_like(C)), length, diam),
                     torch.zeros_like(C))
    d_dev = torch.as_tensor(d_np, device=dev)
    rh_dev = torch.as_tensor(rh_np, device=dev)
    r_dev = s.r_hw.clone()
    ke_dev = s.node_ke_default.clone()
    stream = torch.cuda.current_stream(dev)

    def step(D, R, KE, RH=None, full=False):
        D = D.detach().requires_grad_(True)
        R = R.detach().requires_grad_(True)
        KE = KE.detach().requires_grad_(True)
        h, q, e = implicit_solve(s, D, rh_dev if RH is None else RH, ke=KE, r_hw=R,
                                 accuracy=ACCURACY, polish_steps=POLISH, status_machine=True)
        loss = (h.index_select(1, sens) ** 2).sum()
        loss.backward()
        gR, gK = R.grad, KE.grad
        allreduce_batch_summed([gR, gK])
        gC = gR * dC
        if full:   # the plugin call's whole result: state and gradients
            return loss.detach(), D.grad, gC, gK, h.detach(), q.detach()
        return loss.detach(), D.grad, gC, gK

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        step(d_dev, r_dev, ke_dev)
    barrier()
    # ---- device-timed region: inputs resident in HBM, L2 flushed between steps
    s.launch_events = []
    step_ms = []
    with ClockSampler(_gpu_id_for(local)) as clk:
        barrier()
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            loss, gD, gC, gK = step(d_dev, r_dev, ke_dev)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            step_ms.append(e0.elapsed_time(e1))
        barrier()
    events = s.launch_events
    s.launch_events = None
    total_ms = float(sum(step_ms))
    if world > 1:
        t = torch.tensor([total_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t)
    value = world * B * args.steps / (total_ms / 1e3)
    fwd_ms = [a.elapsed_time(b) for (nm, a, b) in events if nm == "forward"]
    adj_ms = [a.elapsed_time(b) for (nm, a, b) in events if nm == "adjoint"]
    # ---- end to end through the public API with host buffers
    # every input of the call goes host -> device (demand, reservoir heads,
    # roughness-derived resistances, emitter coefficients), and the whole
    # result comes back: loss, gradients w.r.t. demand, C and Ke, heads, flows
    d_host = torch.as_tensor(d_np).pin_memory()
    rh_host = torch.as_tensor(rh_np).pin_memory()
    r_host = r_dev.cpu().pin_memory()
    ke_host = ke_dev.cpu().pin_memory()
    def host_outs():
        return [torch.empty(1, dtype=torch.float64).pin_memory(),
                torch.empty(B, net.N, dtype=torch.float64).pin_memory(),
                torch.empty(net.L, dtype=torch.float64).pin_memory(),
                torch.empty(net.N, dtype=torch.float64).pin_memory(),
                torch.empty(B, net.N, dtype=torch.float64).pin_memory(),
                torch.empty(B, net.L, dtype=torch.float64).pin_memory()]

    outs = host_outs()
    # (1) serial: each step copies its inputs in, runs, copies its result out
    serial_ms = []
    barrier()
    for i in range(args.warmup + args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        Dd = d_host.to(dev, non_blocking=True)
        RHd = rh_host.to(dev, non_blocking=True)
        Rd = r_host.to(dev, non_blocking=True)
        KEd = ke_host.to(dev, non_blocking=True)
        loss, gD, gC, gK, hh, qq = step(Dd, Rd, KEd, RH=RHd, full=True)
        for o, g in zip(outs, (loss.reshape(1), gD, gC, gK, hh, qq)):
            o.copy_(g, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            serial_ms.append(e0.elapsed_time(e1))
    # (2) pipelined, as a serving loop runs the same calls: step i+1's inputs
    # go host -> device on a copy stream while step i computes, and step i's
    # result comes back on that stream while step i+1 computes.  One event
    # pair spans all steps, from the first input copy to the last result
    # copy; the L2 flush between steps stays inside the timed region.
    cs = torch.cuda.Stream(dev)
    obufs = [outs, host_outs()]

    def h2d():
        with torch.cuda.stream(cs):
            xs = [h.to(dev, non_blocking=True) for h in (d_host, rh_host, r_host, ke_host)]
            ev = torch.cuda.Event()
            ev.record(cs)
        return xs, ev

    def pipelined(n_steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        cs.wait_event(e0)
        nxt = h2d()
        for i in range(n_steps):
            xs, ev = nxt
            stream.wait_event(ev)
            for x in xs:
                x.record_stream(stream)
            if i + 1 < n_steps:
                nxt = h2d()
            flush.fill_(1.0)
            res = step(xs[0], xs[2], xs[3], RH=xs[1], full=True)
            done = torch.cuda.Event()
            done.record(stream)
            cs.wait_event(done)
            with torch.cuda.stream(cs):
                for o, g in zip(obufs[i % 2], (res[0].reshape(1),) + tuple(res[1:])):
                    g.record_stream(cs)
                    o.copy_(g, non_blocking=True)
        end = torch.cuda.Event()
        end.record(cs)
        stream.wait_event(end)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1)

    barrier()
    pipelined(args.warmup)
    barrier()
    e2e_total = pipelined(args.steps)
    serial_total = float(sum(serial_ms))
    if world > 1:
        t = torch.tensor([e2e_total, serial_total], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_total, serial_total = float(t[0]), float(t[1])
    h2d = sum(x.numel() * 8 for x in (d_host, rh_host, r_host, ke_host))
    d2h = sum(o.numel() * 8 for o in outs)
    # ---- roofline of the dominant kernel (the fused forward)
    st = s.plan_stats(B)
    iters = s.run(d_dev, rh_dev, ke_dev.unsqueeze(0), r_dev.unsqueeze(0), B, 200, ACCURACY,
                  True, POLISH)["iters"].double()
    # GGA iterations counted without refinement (the band refines only the
    # last one or two of them, so this is a lower bound); polish steps and
    # the terminal factor with two refinements
    rg = s.refine_steps(ACCURACY) if s.refine_band(ACCURACY) <= 0.0 else 0
    bpi = bytes_per_iteration(net.L, st["nnz_A_lower"], st["nnz_L"], st["Nj"], refine=rg)
    bpi2 = bytes_per_iteration(net.L, st["nnz_A_lower"], st["nnz_L"], st["Nj"])
    fwd_bytes = float(iters.sum()) * bpi + B * (POLISH + 1) * bpi2
    fwd_avg_ms = statistics.mean(fwd_ms) if fwd_ms else float("nan")
    adj_avg_ms = statistics.mean(adj_ms) if adj_ms else float("nan")
    dominant = "k_forward" if fwd_avg_ms >= adj_avg_ms else "k_adjoint"
    peak, peak_kind = measured_peak()
    achieved = fwd_bytes / (fwd_avg_ms / 1e3) / 1e9
    traffic_per_scen = read_profile_traffic()
    if world > 1:
        dist.barrier()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD.replace("B=1024", "B=%d" % B), "B": B,
                       "network": "782 jn / 908 links",
                       "l2": "flushed between steps (256 MB write, outside the timed events)",
                       "parallelism": "scenario shards per rank" if world > 1 else "single GPU",
                       "nnz_L": st["nnz_L"], "levels": st["n_levels"],
                       "mean_gga_iters": float(iters.mean())},
            "e2e": {"value": world * B * args.steps / (e2e_total / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "mode": "pipelined: next step's inputs and this step's result copied on a "
                            "second stream while the steps compute; L2 flush inside the timed region",
                    "serial_value": world * B * args.steps / (serial_total / 1e3)},
            "gpu_launches": 2 * args.steps,
            "kernel_ms": {"k_forward": fwd_avg_ms, "k_adjoint": adj_avg_ms},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": peak_kind,
                         "traffic": (traffic_per_scen * B if traffic_per_scen else None),
                         "algorithmic_bytes": fwd_bytes,
                         "model": "bytes/iter = 64L + (16+8r) nA + (3+2r) 8 nL + (32+32r) Nj, r refinements: "
                                  "%d B at r=%d x GGA iters + %d B at r=2 x %d (polish + terminal) per scenario"
                                  % (bpi, rg, bpi2, POLISH + 1)},
            "clocks": clk.summary(),
        }
        if args.workload == "config4":
            line["metric"] = ("fwd+adjoint scenarios/s at B=16384 (782 jn), FP64 factor; "
                              "FP32 factor + FP64 refinement form beside it")
            line["config"]["workload"] = ("large batch: " + line["config"]["workload"])
            line["fp32_form"] = fp32_form(s.net, d_dev, rh_dev, sens, B)
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline_single()
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
