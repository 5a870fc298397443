"""Generate the golden fixtures under tests/golden/ from the reference itself.

Runs only where the reference package (`dgga`) is importable from the
directory named by the REFERENCE_ROOT environment variable (required); the
fixtures it writes are small
.npz files that travel with the tests.  The reference imports `wntr` at module
top for its INP parser only; that package is absent offline, so a stub with
the imported names is placed in sys.modules (the parser is never called: the
networks are built by wdsgpu_b200.synth and handed over field by field).

For each case the fixture stores the network (every Net field), the inputs,
and the reference outputs of
  * GGASolver(mode="dense", dense_status_machine=...).solve(...)   (forward)
  * implicit_solve(..., adjoint="gpu") run on CPU                  (polished
    state and the gradients of a sum-of-squared-heads loss)
  * for small cases, implicit_solve(..., adjoint="cpu") on mode="epanet"
    (the EPANET-replica path with the scipy splu adjoint).

Usage:  REFERENCE_ROOT=<dir> python tests/golden/make_golden.py   (steady cases)
        python tests/golden/make_golden.py eps    (extended-period pin, eps_ref.npz)
        python tests/golden/make_golden.py eps_events (small tanks that fill: shortened
                                                   steps, tank links and a pump changing
                                                   status, eps_events_ref.npz)
        python tests/golden/make_golden.py sens   (sensitivity-matrix pin, sens_ref.npz)
        python tests/golden/make_golden.py pumps  (pump-parameter gradient pins, pump_ref.npz
                                                   and chp_ref.npz)
        python tests/golden/make_golden.py fcv    (flow control valve pin, fcv_ref.npz)
        python tests/golden/make_golden.py psv    (pressure sustaining valve pin, psv_ref.npz)
        python tests/golden/make_golden.py cfg2_wide (config 2, 24 scenarios, cfg2_wide.npz)
        python tests/golden/make_golden.py unrolled (unrolled-K gradient pin, unrolled_ref.npz)
        python tests/golden/make_golden.py unrolled_warm (warm start and frozen statuses,
                                                   unrolled_warm_ref.npz)
        python tests/golden/make_golden.py valves (8 PRVs + 2 PSVs on one network, valves_ref.npz)
        python tests/golden/make_golden.py contract (diag_ratio and record_schedule of solve(),
                                                   contract_ref.npz)
        python tests/golden/make_golden.py cfg3   (the mixed-size workload's 100-junction and
                                                   79-TCV networks, cfg3_small.npz / cfg3_tcv.npz)
"""
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE_ROOT = os.environ.get("REFERENCE_ROOT")


def _install_wntr_stub():
    if "wntr" in sys.modules:
        return
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


def _load_reference():
    if not REFERENCE_ROOT:
        raise SystemExit("set REFERENCE_ROOT to the directory that holds the reference's dgga")
    _install_wntr_stub()
    sys.path.insert(0, REFERENCE_ROOT)
    import dgga.autodiff
    import dgga.parse
    import dgga.solver
    return dgga


def pack_net(net):
    """Net -> flat dict of arrays for np.savez (lists/meta as JSON strings)."""
    out = {}
    for k, v in net.as_fields().items():
        if k in ("node_id", "link_id", "pattern_ids", "meta", "controls_raw",
                 "rules_raw"):
            out["net__" + k] = np.array(json.dumps(v))
        elif k == "patterns":
            out["net__patterns"] = np.array(json.dumps([list(map(float, p)) for p in v]))
        else:
            out["net__" + k] = np.asarray(v)
    return out


def run_case(dgga, torch, net, d, rh, ke, sensors, accuracy, status_machine,
             with_epanet, polish_steps=3):
    ref_net = dgga.parse.Net(**net.as_fields())
    sd = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense",
                               dense_status_machine=status_machine)
    res = {}
    D = torch.tensor(d)
    RH = torch.tensor(rh)
    KE = torch.tensor(ke)
    f = sd.solve(D, RH, ke_int=KE, status_machine=status_machine,
                 accuracy=accuracy, assemble="csr", linear_solver="dense")
    res["fwd_head"] = f["head_ft"].numpy()
    res["fwd_flow"] = f["flow_cfs"].numpy()
    res["fwd_emitter"] = f["emitter_cfs"].numpy()
    res["fwd_iters"] = f["iters"].numpy()
    res["fwd_relerr"] = f["relerr"].numpy()
    res["fwd_converged"] = f["converged"].numpy()
    if "status" in f:
        res["fwd_status"] = f["status"].numpy()
    # implicit solve + adjoint (GPU-route algorithm, run on CPU)
    Dg = D.clone().requires_grad_(True)
    KEg = torch.tensor(ke[0] if ke.ndim == 2 else ke).requires_grad_(True)
    Rg = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
    h, q, e = dgga.autodiff.implicit_solve(
        sd, Dg, RH, ke=KEg, r_hw=Rg, accuracy=accuracy, polish_steps=polish_steps,
        adjoint="gpu", status_machine=status_machine, assemble="csr",
        linear_solver="dense")
    loss = (h[:, sensors] ** 2).sum()
    loss.backward()
    res["imp_head"] = h.detach().numpy()
    res["imp_flow"] = q.detach().numpy()
    res["imp_emitter"] = e.detach().numpy()
    res["grad_demand"] = Dg.grad.numpy()
    res["grad_ke"] = KEg.grad.numpy()
    res["grad_r"] = Rg.grad.numpy()
    res["loss"] = np.array(float(loss))
    if with_epanet:
        se = dgga.solver.GGASolver(ref_net, device="cpu", mode="epanet")
        De = D.clone().requires_grad_(True)
        KEe = torch.tensor(ke[0] if ke.ndim == 2 else ke).requires_grad_(True)
        Re = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
        he, qe, ee = dgga.autodiff.implicit_solve(
            se, De, RH, ke=KEe, r_hw=Re, accuracy=accuracy, adjoint="cpu")
        (he[:, sensors] ** 2).sum().backward()
        res["cpu_head"] = he.detach().numpy()
        res["cpu_flow"] = qe.detach().numpy()
        res["cpu_grad_demand"] = De.grad.numpy()
        res["cpu_grad_ke"] = KEe.grad.numpy()
        res["cpu_grad_r"] = Re.grad.numpy()
    return res


def main():
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    cases = {}
    # config 1: 31 junctions, plain steady GGA (no status machine needed)
    net = synth.config1_network()
    d0 = net.demand_cfs_at(0)
    d = np.stack([d0 * f for f in (0.9, 1.0, 1.1)])
    rh = np.broadcast_to(net.reservoir_head_ft_at(0), d.shape).copy()
    ke = np.broadcast_to(net.node_ke, d.shape).copy()
    sens = synth.sensor_nodes(net, 5)
    cases["cfg1"] = (net, d, rh, ke, sens, 1e-9, False, True)
    # config 2: 782 junctions, 3 PRVs, 20 emitters, status machine
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 4, seed=11)
    ke = np.broadcast_to(net.node_ke, d.shape).copy()
    sens = synth.sensor_nodes(net, 30)
    cases["cfg2"] = (net, d, rh, ke, sens, 1e-6, True, False)
    # every element of the batched path, tank mid-range and at its bottom
    for tag, lvl in (("feat_mid", 0.5), ("feat_low", 0.0)):
        net = synth.feature_network(tank_level=lvl)
        d, _ = synth.config2_scenarios(net, 6, seed=3, sigma=0.4)
        rh = np.broadcast_to(net.fixed_head_ft_at(0), d.shape).copy()
        ke = np.broadcast_to(net.node_ke, d.shape).copy()
        sens = synth.sensor_nodes(net, 6)
        cases[tag] = (net, d, rh, ke, sens, 1e-7, True, False)
    write_cases(dgga, torch, cases)


def write_cases(dgga, torch, cases):
    """Run the reference on each case and write <tag>.npz."""
    for tag, (net, d, rh, ke, sens, acc, sm, ep) in cases.items():
        res = run_case(dgga, torch, net, d, rh, ke, sens, acc, sm, ep)
        blob = pack_net(net)
        blob.update({"in_demand": d, "in_res_head": rh, "in_ke": ke,
                     "in_sensors": np.asarray(sens), "in_accuracy": np.array(acc),
                     "in_status_machine": np.array(sm)})
        blob.update({"ref_" + k: v for k, v in res.items()})
        path = os.path.join(HERE, tag + ".npz")
        np.savez_compressed(path, **blob)
        print("%-9s iters=%s -> %s (%d KB)" % (
            tag, res["fwd_iters"].tolist(), os.path.basename(path),
            os.path.getsize(path) // 1024))


def make_cfg2_wide():
    """Config 2 at 24 scenarios with a wider demand spread (lognormal 0.35,
    seed 12): more scenarios of the headline network, more PRV status
    changes, pinned to the reference like cfg2."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 24, seed=12, sigma=0.35)
    ke = np.broadcast_to(net.node_ke, d.shape).copy()
    sens = synth.sensor_nodes(net, 30)
    write_cases(dgga, torch, {"cfg2_wide": (net, d, rh, ke, sens, 1e-6, True, False)})


def make_cfg3():
    """The mixed-size workload's own networks, pinned one by one: the
    100-junction looped network and the 542-junction network with 79 throttle
    control valves (the Km / CSMALL valve branch, dgga/solver.py:2203-2219),
    four scenarios each at the workload's lognormal(0.3) demand spread, with
    the status machine."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    nets = synth.config3_networks()
    cases = {}
    for tag, net, seed in (("cfg3_small", nets[0], 61), ("cfg3_tcv", nets[1], 62)):
        d, _ = synth.config2_scenarios(net, 4, seed=seed, sigma=0.3)
        rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
        ke = np.broadcast_to(net.node_ke, d.shape).copy()
        sens = synth.sensor_nodes(net, 8)
        cases[tag] = (net, d, rh, ke, sens, 1e-6, True, False)
    write_cases(dgga, torch, cases)


def make_eps(T=6, name="eps_ref", tank_range_m=10.0, tank_diam_m=(15.0, 30.0)):
    """Extended-period pin: the reference's serial EPANET-replica EpsDriver
    (dgga/eps.py) on a small pump/tank network, one scenario, T hourly
    demand periods (duration (T - 1) hours).  The scenario's noisy diurnal
    demands are given to the reference as one demand pattern per junction.
    Tank mid-range heads come from a reference steady solve with the tank
    nodes as zero-demand junctions.  `eps` keeps the tanks inside their
    range (hourly frames); `eps_events` uses small tanks (2 m range, 4-6 m
    across) that fill within the run, so EpsDriver shortens steps at tank
    fill/empty times, tank links close and reopen (tankstatus) and a pump
    goes from XHEAD to open: eps_events_ref.npz."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    from wdsgpu_b200.net import JUNCTION, Net
    dgga = _load_reference()
    import dgga.eps
    torch.set_default_dtype(torch.float64)
    net0 = synth.eps_network(seed=7)
    tn = np.asarray(net0.tank_node)
    f = dict(net0.as_fields())
    nt = np.asarray(f["node_type"]).copy()
    nt[tn] = JUNCTION
    jn = np.flatnonzero(nt == JUNCTION)
    d0 = net0.demand_cfs_at(0)
    empty = dict(tank_node=np.zeros(0, np.int32), tank_overflow=np.zeros(0, np.int8))
    for k in ("tank_h0", "tank_hmin", "tank_hmax", "tank_area", "tank_vmin", "tank_v0",
              "tank_vmax"):
        empty[k] = np.zeros(0)
    f.update(node_type=nt, dem_node=jn.astype(np.int32), dem_base_cfs=d0[jn],
             dem_pat=np.full(jn.size, -1, np.int32), **empty)
    pre = dgga.solver.GGASolver(dgga.parse.Net(**f), device="cpu", mode="dense",
                                dense_status_machine=True)
    o = pre.solve(torch.tensor(d0[None]), torch.tensor(np.nan_to_num(Net(**f).fixed_head_ft_at(0))[None]),
                  status_machine=True, accuracy=1e-8, assemble="csr", linear_solver="dense")
    centers = o["head_ft"][0].numpy()[tn]
    net = synth.eps_network(seed=7, tank_center_ft=centers, tank_range_m=tank_range_m,
                            tank_diam_m=tank_diam_m)
    dem = synth.eps_demands(net, T, 1, seed=3)           # [T, 1, N] cfs
    # one pattern per junction reproduces dem[t, 0, node] = base * factor[t]
    fl = dict(net.as_fields())
    junc = np.asarray(fl["dem_node"])
    base = np.asarray(fl["dem_base_cfs"])
    pats = [list(map(float, dem[:, 0, n] / b)) for n, b in zip(junc, base)]
    fl.update(patterns=pats, pattern_ids=["p%d" % i for i in range(len(pats))],
              dem_pat=np.arange(junc.size, dtype=np.int32))
    meta = dict(fl["meta"])
    meta.update(duration_sec=(T - 1) * 3600, hyd_step_sec=3600, pat_step_sec=3600,
                report_step_sec=3600, pat_start_sec=0, tstart_sec=0, accuracy=1e-5)
    fl["meta"] = meta
    ref_net = dgga.parse.Net(**fl)
    frames = dgga.eps.EpsDriver(ref_net).run()
    blob = pack_net(net)
    blob.update({"in_demand": dem, "in_T": np.array(T)})
    for k in ("t_sec", "head_ft", "flow_int_cfs", "status", "iterations", "relerr"):
        blob["ref_" + k] = np.asarray(frames[k])
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **blob)
    print("%s: frames at t=%s, iterations %s -> %s" % (
        name, frames["t_sec"].tolist(), frames["iterations"].tolist(), os.path.basename(path)))


def make_sens():
    """Sensitivity pin: the reference's sensitivity_matrix (dgga/sensitivity.py:
    59-145, one splu per frame and m sensor columns, EPANET-replica mode) on
    the config-2 network, two frames, six sensors, w.r.t. C and w.r.t. r."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    import dgga.sensitivity
    torch.set_default_dtype(torch.float64)
    net = synth.config2_network()
    d, rh = synth.config2_scenarios(net, 2, seed=61)
    sens = synth.sensor_nodes(net, 6, seed=9)
    ref_net = dgga.parse.Net(**net.as_fields())
    # mode="epanet": the reference's polished solve runs the status machine
    # there (its dense mode refuses PRV networks without it)
    sd = dgga.solver.GGASolver(ref_net, device="cpu", mode="epanet")
    r = np.asarray(net.r_hw, dtype=np.float64)
    # device statuses of each frame from the reference's own batched status
    # machine (sensitivity_matrix freezes the statuses it is given)
    dn = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense", dense_status_machine=True)
    st = dn.solve(torch.tensor(d), torch.tensor(rh), status_machine=True, accuracy=1e-10,
                  assemble="csr", linear_solver="dense")["status"].numpy()
    res = {"status": st}
    for wrt in ("C", "r"):
        blocks = []
        for b in range(d.shape[0]):
            S = dgga.sensitivity.sensitivity_matrix(
                sd, torch.tensor(d[b:b + 1]), torch.tensor(rh[b:b + 1]), torch.tensor(r), sens,
                wrt=wrt, accuracy=1e-10, status=st[b])
            blocks.append(np.asarray(S))
        res["S_" + wrt] = np.concatenate(blocks, axis=0)
    blob = pack_net(net)
    blob.update({"in_demand": d, "in_res_head": rh, "in_sensors": np.asarray(sens)})
    blob.update({"ref_" + k: v for k, v in res.items()})
    path = os.path.join(HERE, "sens_ref.npz")
    np.savez_compressed(path, **blob)
    print("sens: S_C %s, max |S_C| %.3g -> %s" % (res["S_C"].shape, np.abs(res["S_C"]).max(),
                                                  os.path.basename(path)))


def _pump_case(dgga, torch, net, d, rh, speed_scale, h0_scale, r_scale, name):
    """The reference's CPU implicit adjoint with pump theta (ImplicitGGASolve,
    dgga/autodiff.py:609-756: speed / pump_h0 / pump_r as differentiable [L]
    tensors, statuses frozen), one scenario per call (the statuses are per
    scenario), each scenario given the statuses of the reference's own dense
    status machine.  The loss is the sum of squared heads at the sensors and
    at the pumps' downstream nodes plus the sum of squared pump flows."""
    ke = np.asarray(net.node_ke, dtype=np.float64)
    sens = synth_sensor_nodes(net)
    ref_net = dgga.parse.Net(**net.as_fields())
    se = dgga.solver.GGASolver(ref_net, device="cpu", mode="epanet")
    pl = np.asarray(net.pump_link, dtype=np.int64)
    pn2 = np.asarray(net.link_n2, dtype=np.int64)[pl]
    speed = np.asarray(se.init_setting, dtype=np.float64).copy()
    speed[pl] = speed[pl] * np.asarray(speed_scale)
    h0 = np.asarray(se.pl_h0, dtype=np.float64).copy()
    h0[pl] = h0[pl] * np.asarray(h0_scale)
    rp = np.asarray(se.pl_r, dtype=np.float64).copy()
    rp[pl] = rp[pl] * np.asarray(r_scale)
    dn = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense", dense_status_machine=True)
    st = dn.solve(torch.tensor(d), torch.tensor(rh), status_machine=True, accuracy=1e-10,
                  assemble="csr", linear_solver="dense")["status"].numpy()
    keys = ("head", "flow", "g_speed", "g_h0", "g_r", "g_demand", "g_rhw", "g_res_head")
    res = {k: [] for k in keys}
    for b in range(d.shape[0]):
        D = torch.tensor(d[b:b + 1]).requires_grad_(True)
        RH = torch.tensor(rh[b:b + 1]).requires_grad_(True)
        R = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
        sp = torch.tensor(speed).requires_grad_(True)
        h0t = torch.tensor(h0).requires_grad_(True)
        rpt = torch.tensor(rp).requires_grad_(True)
        h, q, e = dgga.autodiff.implicit_solve(
            se, D, RH, ke=torch.tensor(ke), r_hw=R, accuracy=1e-10,
            adjoint="cpu", speed=sp, pump_h0=h0t, pump_r=rpt, status=st[b])
        loss = (h[:, sens] ** 2).sum() + (h[:, pn2] ** 2).sum() + (q[:, pl] ** 2).sum()
        loss.backward()
        for k, v in zip(keys, (h.detach(), q.detach(), sp.grad, h0t.grad, rpt.grad, D.grad,
                               R.grad, RH.grad)):
            res[k].append(np.asarray(v).reshape(-1))
    blob = pack_net(net)
    blob.update({"in_demand": d, "in_res_head": rh, "in_ke": ke, "in_sensors": np.asarray(sens),
                 "in_speed": speed, "in_pump_h0": h0, "in_pump_r": rp, "in_status": st})
    blob.update({"ref_" + k: np.stack(v) for k, v in res.items()})
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **blob)
    print("%s: g_speed at pumps %s -> %s" % (
        name, np.stack(res["g_speed"])[:, pl].tolist(), os.path.basename(path)))


def synth_sensor_nodes(net):
    from wdsgpu_b200 import synth
    return synth.sensor_nodes(net, 6)


def make_pumps():
    """Pump-parameter pins.  pump_ref: the feature network with all four pump
    kinds (power function, custom curve, no curve, constant HP) at speeds and
    curve coefficients moved off the network's values.  chp_ref: the same
    network with its constant-HP pump feeding a dead end of tiny demand, so
    that the pump sits on its CBIG clamp branch (hydcoeffs.c:748-752) at the
    converged state."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.feature_network(tank_level=0.5, with_chp=True)
    d, _ = synth.config2_scenarios(net, 3, seed=17, sigma=0.3)
    rh = np.broadcast_to(net.fixed_head_ft_at(0), d.shape).copy()
    _pump_case(dgga, torch, net, d, rh, [0.97, 1.04, 1.0, 1.02], [1.03, 1, 1, 1],
               [0.95, 1, 1, 1.05], "pump_ref")
    net = synth.chp_dead_end_network()
    d, _ = synth.config2_scenarios(net, 3, seed=17, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    _pump_case(dgga, torch, net, d, rh, [0.97, 1.0, 1.0, 1.02], [1, 1, 1, 1],
               [1, 1, 1, 1.05], "chp_ref")


def _valve_case(dgga, torch, net, d, rh, links, name):
    """The reference's EPANET replica (mode="epanet", status_machine=True,
    dgga/solver.py:1922-2130) per scenario, then its CPU implicit adjoint
    (ImplicitGGASolve, dgga/autodiff.py:609-756) with that scenario's final
    statuses frozen, for L = sum of squared sensor heads + squared flows of
    the given valve links."""
    from wdsgpu_b200 import synth
    ke = np.asarray(net.node_ke, dtype=np.float64)
    sens = synth.sensor_nodes(net, 6)
    ref_net = dgga.parse.Net(**net.as_fields())
    se = dgga.solver.GGASolver(ref_net, device="cpu", mode="epanet")
    keys = ("fwd_head", "fwd_flow", "fwd_status", "fwd_iters", "head", "flow", "g_demand",
            "g_ke", "g_rhw", "g_res_head")
    res = {k: [] for k in keys}
    for b in range(d.shape[0]):
        f = se.solve(torch.tensor(d[b:b + 1]), torch.tensor(rh[b:b + 1]),
                     ke_int=torch.tensor(ke[None]), accuracy=1e-7, status_machine=True)
        st = np.asarray(f["status"]).reshape(-1)
        D = torch.tensor(d[b:b + 1]).requires_grad_(True)
        RH = torch.tensor(rh[b:b + 1]).requires_grad_(True)
        KE = torch.tensor(ke).requires_grad_(True)
        R = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
        h, q, e = dgga.autodiff.implicit_solve(se, D, RH, ke=KE, r_hw=R, accuracy=1e-10,
                                               adjoint="cpu", status=st)
        loss = (h[:, sens] ** 2).sum() + (q[:, links] ** 2).sum()
        loss.backward()
        for k, v in zip(keys, (f["head_ft"], f["flow_cfs"], st, f["iters"], h.detach(),
                               q.detach(), D.grad, KE.grad, R.grad, RH.grad)):
            res[k].append(np.asarray(v).reshape(-1))
    blob = pack_net(net)
    blob.update({"in_demand": d, "in_res_head": rh, "in_ke": ke, "in_sensors": np.asarray(sens),
                 "in_loss_links": np.asarray(links)})
    blob.update({"ref_" + k: np.stack(v) for k, v in res.items()})
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **blob)
    print("%s: iters %s, valve statuses %s -> %s" % (
        name, np.stack(res["fwd_iters"]).ravel().tolist(),
        np.stack(res["fwd_status"])[:, links].tolist(), os.path.basename(path)))


def make_fcv():
    """FCV pin: the feature network with two FCVs, one throttling (ACTIVE) and
    one pushed beyond what the network delivers (XFCV), four scenarios
    (fcvcoeff, fcvstatus in linkstatus, valve-order Xflow of the replica)."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.fcv_network()
    d, _ = synth.config2_scenarios(net, 4, seed=23, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    _valve_case(dgga, torch, net, d, rh, np.flatnonzero(np.asarray(net.link_type) == 6),
                "fcv_ref")


def make_psv():
    """PSV pin: the feature network (ACTIVE PRV) plus a PSV that throttles to
    hold its upstream pressure, four scenarios (psvcoeff, psvstatus in
    valvestatus); the loss takes both valves' flows, so the adjoint's
    constraint rows of both orientations carry a right-hand side."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.psv_network()
    d, _ = synth.config2_scenarios(net, 4, seed=29, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    lt = np.asarray(net.link_type)
    _valve_case(dgga, torch, net, d, rh, np.flatnonzero((lt == 3) | (lt == 4)), "psv_ref")


def make_valves():
    """Many-valve pin: eight PRV zones and two PSVs on one 520-junction
    network, four scenarios, every valve ACTIVE in most of them (ten
    constraint rows in the polish and the adjoint; the reference's valve loop
    and Woodbury take any count, dgga/solver.py:863, dgga/autodiff.py:
    965-1029).  The EPANET replica with its status machine and the CPU
    adjoint, as for the PSV pin (the reference's dense route refuses PSVs)."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.many_valves_network()
    d, _ = synth.config2_scenarios(net, 4, seed=31, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    lt = np.asarray(net.link_type)
    _valve_case(dgga, torch, net, d, rh, np.flatnonzero((lt == 3) | (lt == 4)), "valves_ref")


def make_contract():
    """The rest of solve()'s result contract on the golden inputs: the
    condition proxy `diag_ratio` (dgga/solver.py:3026-3032, 3205-3207) and
    the status-machine schedule of record_schedule=True (:2740-2745,
    3154-3160), from the reference's dense batched route, for the cfg2,
    feat_mid, feat_low and cfg3_tcv cases.  Writes contract_ref.npz with
    <tag>__diag_ratio and <tag>__sched_{it,valve,a,b,chg} arrays (one row per
    schedule entry: a valve-pass entry has valve = True, a = act; a
    link-status entry a = conv, b = per)."""
    import torch
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.dirname(HERE))
    from golden.load import load
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    blob = {}
    for tag in ("cfg2", "feat_mid", "feat_low", "cfg3_tcv"):
        net, inp, _ = load(tag)
        ref_net = dgga.parse.Net(**net.as_fields())
        sd = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense",
                                   dense_status_machine=True)
        f = sd.solve(torch.tensor(inp["demand"]), torch.tensor(inp["res_head"]),
                     ke_int=torch.tensor(inp["ke"]), status_machine=True,
                     accuracy=float(inp["accuracy"]), assemble="csr", linear_solver="dense",
                     record_schedule=True)
        if "diag_ratio" in f:
            blob[tag + "__diag_ratio"] = f["diag_ratio"].numpy()
        sch = f["schedule"]
        B = inp["demand"].shape[0]
        blob[tag + "__sched_it"] = np.array([e["it"] for e in sch], dtype=np.int64)
        blob[tag + "__sched_valve"] = np.array([e.get("kind") == "valve" for e in sch])
        blob[tag + "__sched_a"] = np.stack([np.asarray(e["act"] if e.get("kind") == "valve"
                                                       else e["conv"]) for e in sch]).astype(bool)
        blob[tag + "__sched_b"] = np.stack([np.asarray(e["per"]) if "per" in e
                                            else np.zeros(B, bool) for e in sch]).astype(bool)
        blob[tag + "__sched_chg"] = np.stack([e["chg"] for e in sch]).astype(bool)
        print("%-9s schedule iterations %s, changes %d, diag_ratio %s" % (
            tag, blob[tag + "__sched_it"].tolist(), int(blob[tag + "__sched_chg"].sum()),
            None if "diag_ratio" not in f else f["diag_ratio"].numpy().round(1).tolist()))
    path = os.path.join(HERE, "contract_ref.npz")
    np.savez_compressed(path, **blob)


def make_unrolled():
    """Unrolled-K pin: the reference's solve_unrolled (dgga/autodiff.py:
    1357-1664, K = 8 fixed GGA iterations, statuses frozen at the initial
    configuration, dense mode) and its autograd gradients w.r.t. demand,
    reservoir/tank heads, emitter Ke and pipe resistance, for L = sum of
    squared sensor heads + squared pump flows + squared emitter flows."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.unrolled_network()
    d, _ = synth.config2_scenarios(net, 3, seed=41, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    ke = np.broadcast_to(np.asarray(net.node_ke, dtype=np.float64), d.shape).copy()
    sens = synth.sensor_nodes(net, 6)
    pl = np.asarray(net.pump_link, dtype=np.int64)
    emn = np.flatnonzero(np.asarray(net.node_ke) > 0)
    K = 8
    ref_net = dgga.parse.Net(**net.as_fields())
    # dense_status_machine=True admits the check-valve pipe; solve_unrolled
    # itself freezes the statuses at the initial configuration
    sd = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense", dense_status_machine=True)
    D = torch.tensor(d).requires_grad_(True)
    RH = torch.tensor(rh).requires_grad_(True)
    KE = torch.tensor(ke).requires_grad_(True)
    R = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
    out = dgga.autodiff.solve_unrolled(sd, D, RH, ke=KE, r_hw=R, K=K)
    h, q, e = out["head_ft"], out["flow_cfs"], out["emitter_cfs"]
    loss = (h[:, sens] ** 2).sum() + (q[:, pl] ** 2).sum() + (e[:, emn] ** 2).sum()
    loss.backward()
    blob = pack_net(net)
    blob.update({"in_demand": d, "in_res_head": rh, "in_ke": ke, "in_sensors": np.asarray(sens),
                 "in_K": np.array(K)})
    res = dict(head=h.detach().numpy(), flow=q.detach().numpy(), emitter=e.detach().numpy(),
               g_demand=D.grad.numpy(), g_res_head=RH.grad.numpy(), g_ke=KE.grad.numpy(),
               g_rhw=R.grad.numpy())
    blob.update({"ref_" + k: v for k, v in res.items()})
    path = os.path.join(HERE, "unrolled_ref.npz")
    np.savez_compressed(path, **blob)
    print("unrolled: K=%d, max |g_demand| %.3g -> %s" % (K, np.abs(res["g_demand"]).max(),
                                                         os.path.basename(path)))


def make_unrolled_warm():
    """Unrolled-K pin with a warm start and frozen statuses: the reference's
    solve_unrolled (dgga/autodiff.py:1357-1664) at K = 6 from the flows and
    emitter flows of its own dense solve at 90 % demand (q0 [B,L], e0 [B,N])
    and with the statuses that solve ended with frozen (status [L]), on the
    unrolled feature network."""
    import torch
    sys.path.insert(0, REPO)
    from wdsgpu_b200 import synth
    dgga = _load_reference()
    torch.set_default_dtype(torch.float64)
    net = synth.unrolled_network()
    d, _ = synth.config2_scenarios(net, 3, seed=43, sigma=0.3)
    rh = np.broadcast_to(np.nan_to_num(net.fixed_head_ft_at(0)), d.shape).copy()
    ke = np.broadcast_to(np.asarray(net.node_ke, dtype=np.float64), d.shape).copy()
    sens = synth.sensor_nodes(net, 6)
    pl = np.asarray(net.pump_link, dtype=np.int64)
    emn = np.flatnonzero(np.asarray(net.node_ke) > 0)
    K = 6
    ref_net = dgga.parse.Net(**net.as_fields())
    sd = dgga.solver.GGASolver(ref_net, device="cpu", mode="dense", dense_status_machine=True)
    f = sd.solve(torch.tensor(0.9 * d), torch.tensor(rh), ke_int=torch.tensor(ke),
                 status_machine=True, accuracy=1e-6, assemble="csr", linear_solver="dense")
    q0 = f["flow_cfs"].numpy()
    e0 = f["emitter_cfs"].numpy()
    st = f["status"].numpy()[0].astype(np.int8)
    D = torch.tensor(d).requires_grad_(True)
    RH = torch.tensor(rh).requires_grad_(True)
    KE = torch.tensor(ke).requires_grad_(True)
    R = torch.tensor(np.asarray(net.r_hw, dtype=np.float64)).requires_grad_(True)
    out = dgga.autodiff.solve_unrolled(sd, D, RH, ke=KE, r_hw=R, K=K, q0=torch.tensor(q0),
                                       e0=torch.tensor(e0), status=st)
    h, q, e = out["head_ft"], out["flow_cfs"], out["emitter_cfs"]
    loss = (h[:, sens] ** 2).sum() + (q[:, pl] ** 2).sum() + (e[:, emn] ** 2).sum()
    loss.backward()
    blob = pack_net(net)
    blob.update({"in_demand": d, "in_res_head": rh, "in_ke": ke, "in_sensors": np.asarray(sens),
                 "in_K": np.array(K), "in_q0": q0, "in_e0": e0, "in_status": st})
    res = dict(head=h.detach().numpy(), flow=q.detach().numpy(), emitter=e.detach().numpy(),
               g_demand=D.grad.numpy(), g_res_head=RH.grad.numpy(), g_ke=KE.grad.numpy(),
               g_rhw=R.grad.numpy())
    blob.update({"ref_" + k: v for k, v in res.items()})
    path = os.path.join(HERE, "unrolled_warm_ref.npz")
    np.savez_compressed(path, **blob)
    print("unrolled_warm: K=%d, statuses %s -> %s" % (K, np.bincount(st).tolist(),
                                                      os.path.basename(path)))


if __name__ == "__main__":
    if sys.argv[1:] == ["eps"]:
        make_eps()
    elif sys.argv[1:] == ["eps_events"]:
        make_eps(T=9, name="eps_events_ref", tank_range_m=2.0, tank_diam_m=(4.0, 6.0))
    elif sys.argv[1:] == ["sens"]:
        make_sens()
    elif sys.argv[1:] == ["pumps"]:
        make_pumps()
    elif sys.argv[1:] == ["fcv"]:
        make_fcv()
    elif sys.argv[1:] == ["psv"]:
        make_psv()
    elif sys.argv[1:] == ["unrolled"]:
        make_unrolled()
    elif sys.argv[1:] == ["unrolled_warm"]:
        make_unrolled_warm()
    elif sys.argv[1:] == ["cfg2_wide"]:
        make_cfg2_wide()
    elif sys.argv[1:] == ["cfg3"]:
        make_cfg3()
    elif sys.argv[1:] == ["valves"]:
        make_valves()
    elif sys.argv[1:] == ["contract"]:
        make_contract()
    else:
        main()
