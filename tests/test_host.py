"""Host-side admission rules and error classes of GGASolver / implicit_solve
(mirroring dgga/solver.py:160-495 and dgga/autodiff.py:1315-1351).  CPU only:
the constructor builds the tables without touching the device."""
import copy

import numpy as np
import pytest
import torch

from wdsgpu_b200 import synth
from wdsgpu_b200.autodiff import dr_dC, hw_resistance, implicit_solve
from wdsgpu_b200.net import FCV, PBV, PSV
from wdsgpu_b200.solver import GGASolver


def test_unsupported_link_types_raise():
    net = synth.feature_network()
    with pytest.raises(NotImplementedError):       # CVPIPE/PRV need the status machine
        GGASolver(net, device="cpu", dense_status_machine=False)
    n2 = copy.deepcopy(net)
    n2.link_type = n2.link_type.copy()
    n2.link_type[0] = PSV                          # batched PSVs (status machine only)
    GGASolver(n2, device="cpu", dense_status_machine=True)
    with pytest.raises(NotImplementedError):
        GGASolver(n2, device="cpu", dense_status_machine=False)
    n2.link_type[0] = PBV
    with pytest.raises(NotImplementedError):
        GGASolver(n2, device="cpu", dense_status_machine=True)
    n2.link_type[0] = FCV                          # batched FCVs (status machine only)
    GGASolver(n2, device="cpu", dense_status_machine=True)
    with pytest.raises(NotImplementedError):
        GGASolver(n2, device="cpu", dense_status_machine=False)


def test_meta_guards():
    for key, val in (("headloss", "D-W"), ("demand_model", "PDA"), ("damp_limit", 0.5),
                     ("headerror", 0.1)):
        net = synth.config1_network()
        net.meta[key] = val
        with pytest.raises(NotImplementedError):
            GGASolver(net, device="cpu")
    with pytest.raises(ValueError):
        GGASolver(synth.config1_network(), mode="bogus")
    with pytest.raises(NotImplementedError):
        GGASolver(synth.config1_network(), mode="epanet")


def test_solve_argument_guards():
    s = GGASolver(synth.config1_network(), device="cpu")
    d, rh = s.net.demand_cfs_at(0), s.net.reservoir_head_ft_at(0)
    with pytest.raises(ValueError):
        s.solve(d, rh, assemble="coo")
    with pytest.raises(ValueError):
        s.solve(d, rh, linear_solver="magma")
    with pytest.raises(NotImplementedError):
        s.solve(d, rh, linear_solver="cudss")
    with pytest.raises(ValueError):
        s.solve(d, rh, assemble="dense", linear_solver="sm100")
    with pytest.raises(NotImplementedError):
        s.solve(d, rh, status_machine=True)       # needs dense_status_machine
    with pytest.raises(ValueError):           # the reference: dense status machine only
        s.solve(d, rh, record_schedule=True)


def test_prv_needs_status_machine_and_float64():
    net = synth.config2_network()
    s = GGASolver(net, device="cpu", dense_status_machine=True)
    with pytest.raises(NotImplementedError):
        s.solve(net.demand_cfs_at(0), net.reservoir_head_ft_at(0), status_machine=False)
    with pytest.raises(NotImplementedError):
        GGASolver(net, device="cpu", dtype=torch.float32, dense_status_machine=True)


def test_implicit_solve_guards():
    s = GGASolver(synth.config1_network(), device="cpu")
    d, rh = s.net.demand_cfs_at(0), s.net.reservoir_head_ft_at(0)
    with pytest.raises(NotImplementedError):
        implicit_solve(s, d, rh, adjoint="cpu")
    with pytest.raises(ValueError):
        implicit_solve(s, d, rh, adjoint="both")
    with pytest.raises(ValueError):                 # pump rows are [L] or [B, L]
        implicit_solve(s, d, rh, speed=np.ones(3))


def test_tables_follow_reference_setup():
    """Per-link tables derived like GGASolver.__init__: TCV Km from the
    setting, PRV setting in ft, initial flows, status codes."""
    net = synth.feature_network()
    s = GGASolver(net, device="cpu", dense_status_machine=True)
    t = s._tables
    lt = np.asarray(net.link_type)
    tcv = np.flatnonzero(lt == 7)
    d = net.diam_ft[tcv]
    np.testing.assert_allclose(t["km_tcv"][tcv], 0.02517 * net.valve_setting_user[tcv] / (d * d * d * d))
    pcv = s.pcv_links
    np.testing.assert_allclose(t["prv_hset"][pcv],
                               net.elev_ft[net.link_n2[pcv]] + net.valve_setting_user[pcv] / 0.3048)
    closed = np.flatnonzero(np.asarray(net.init_status) == 0)
    assert (t["q_init"][closed] == 1e-6).all()
    assert (t["status0"][closed] == 2).all()


def test_roughness_chain_rule():
    C = np.array([100.0, 130.0])
    L = np.array([1000.0, 500.0])
    D = np.array([1.0, 0.5])
    h = 1e-6 * C
    fd = (hw_resistance(C + h, L, D) - hw_resistance(C - h, L, D)) / (2 * h)
    np.testing.assert_allclose(dr_dC(C, L, D), fd, rtol=1e-7)


def test_synthetic_networks_are_seeded():
    a, b = synth.config2_network(), synth.config2_network()
    np.testing.assert_array_equal(a.link_n1, b.link_n1)
    np.testing.assert_array_equal(a.r_hw, b.r_hw)
    assert a.N == 784 and a.L == 908
    assert (np.asarray(a.node_type) == 0).sum() == 782
    assert (np.asarray(a.link_type) == 3).sum() == 3
    assert (np.asarray(a.link_type) == 1).sum() == 905
    assert (a.node_ke > 0).sum() == 20


def test_pump_rows_host_rules():
    """speed / pump_h0 / pump_r rows: [L] or [B,L]; speed equals the
    network's link settings off pump links (the reference's speed sets valve
    settings there, dgga/autodiff.py:99-120)."""
    net = synth.feature_network(with_chp=True)
    s = GGASolver(net, device="cpu", dense_status_machine=True)
    pl = np.asarray(net.pump_link)
    sp = s.init_setting.copy()
    sp[pl] *= 1.05
    rows = s.pump_rows(3, speed=sp)
    assert rows[0].shape == (1, s.L) and rows[1] is None and rows[2] is None
    rows = s.pump_rows(3, speed=sp, pump_h0=np.tile(np.zeros(s.L), (3, 1)))
    assert rows[0].shape == (3, s.L) and rows[1].shape == (3, s.L)
    assert s.pump_rows(3) is None
    with pytest.raises(ValueError):
        s.pump_rows(3, pump_r=np.zeros((2, s.L)))
    bad = sp.copy()
    bad[np.flatnonzero(np.asarray(net.link_type) != 2)[0]] += 1.0   # a non-pump link
    with pytest.raises(NotImplementedError):
        s.pump_rows(3, speed=bad)
    with pytest.raises(NotImplementedError):                         # frozen status
        implicit_solve(s, net.demand_cfs_at(0), net.fixed_head_ft_at(0),
                       status=np.zeros(s.L, dtype=np.int8))


def test_unrolled_host_rules():
    """solve_unrolled refuses what the reference refuses (control valves) and
    what this route does not take (pump parameters); the health probe checks
    its parameter name."""
    from wdsgpu_b200.autodiff import solve_unrolled, unrolled_grad_health
    s = GGASolver(synth.config2_network(), device="cpu", dense_status_machine=True)
    d, rh = s.net.demand_cfs_at(0), s.net.reservoir_head_ft_at(0)
    with pytest.raises(NotImplementedError):          # PRVs with a setting
        solve_unrolled(s, d, rh, K=3)
    s2 = GGASolver(synth.unrolled_network(), device="cpu", dense_status_machine=True)
    with pytest.raises(NotImplementedError):
        solve_unrolled(s2, d, rh, K=3, speed=s2.init_setting.copy())
    with pytest.raises(ValueError):
        solve_unrolled(s2, d, rh, K=3, assemble="dense")
    with pytest.raises(ValueError):
        unrolled_grad_health(s2, d, rh, param="speed")
